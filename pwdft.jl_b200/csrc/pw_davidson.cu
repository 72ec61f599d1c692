// pw_davidson: diag_davidson_qe! for one k-point (diag_davidson_qe_v2.jl:38-216),
// the QE-style block Davidson with Nvecx = 2 Nvec and restart, for
// norm-conserving pseudopotentials (S = identity, so Spsi is psi itself).
// Every block operation runs on the device: the correction vectors
// (H - e) psi vc through pw_rotate, Kprec through pw_kprec, the new H psi
// through pw_apply, the reduced-matrix columns psi' Hpsi_new / psi' psi_new
// through pw_gram (tcgen05 split-BF16x3 for complex64, FP64 CUDA cores for
// complex128), and the generalized eigenproblem of the reduced matrices
// (order nbase <= 2 Nvec, lowest Nvec pairs) through pw_eig.cu's solver.  The
// host only steers: it reads the Nvec Ritz values per iteration for the
// convergence test |ew - evals| < EBANDS_THR and reorders the coefficient
// columns of the unconverged roots, as the reference does.
// Mixed precision: a reduced overlap Sc that the split-BF16 Gram leaves not
// positive definite ends the iteration with the Ritz vectors of the last
// successful step (counted as 1000 x restarts in *niter); the FP64 path
// reports PW_ERR_NOT_POSDEF as the reference's generalized eigen would.
#include <vector>

#include "pw_rr.cuh"

namespace {

// M (n x m, ld n) = V (ld ldv) * diag(-shift): the -e_j psi vc_j part of the
// correction vectors (diag_davidson_qe_v2.jl:107-110) folded into the
// coefficients, so one rotation of psi and one of Hpsi build (H - e) psi vc.
__global__ void k_shift_cols(const double2 *V, int ldv, const double *shift, double2 *M, int n, int m) {
    const size_t total = (size_t)n * m;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        const double2 v = V[(size_t)j * ldv + i];
        const double s = -shift[j];
        M[t] = make_double2(v.x * s, v.y * s);
    }
}

// Upper triangles of Hc and Sc (order n, ld lds) into dense n x n T and G for
// the eigensolver, with real diagonals (diag_davidson_qe_v2.jl:139-149:
// the solver reads the upper triangles only, so this is Hermitian(Hc)).
__global__ void k_take_upper(const double2 *Hc, const double2 *Sc, int lds, double2 *T, double2 *G, int n) {
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        if (i > j) continue;
        double2 h = Hc[(size_t)j * lds + i], s = Sc[(size_t)j * lds + i];
        if (i == j) h.y = s.y = 0.0;
        T[t] = h;
        G[t] = s;
    }
}

// Restart of the reduced problem (diag_davidson_qe_v2.jl:200-208): columns
// 0..nb-1 of Hc, Sc, vc (ld nx) cleared, Hc = diag(evals), Sc = vc = I.
__global__ void k_reset_reduced(double2 *Hc, double2 *Sc, double2 *vc, int nx, int nb, const double *evals) {
    const size_t total = (size_t)nx * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / nx), i = (int)(t - (size_t)j * nx);
        const bool d = i == j;
        Hc[t] = make_double2(d ? evals[j] : 0.0, 0.0);
        Sc[t] = make_double2(d ? 1.0 : 0.0, 0.0);
        vc[t] = make_double2(d ? 1.0 : 0.0, 0.0);
    }
}

// Each column of the block scaled to unit norm, the norm summed in FP64
// (diag_davidson_qe_v2.jl:119-127); one CTA per column.
template <typename C>
__global__ void k_normalize_cols(C *X, int64_t ld, int ngw) {
    __shared__ double red[32];
    C *x = X + (size_t)blockIdx.x * ld;
    double s = 0.0;
    for (int g = threadIdx.x; g < ngw; g += blockDim.x) s += (double)x[g].x * x[g].x + (double)x[g].y * x[g].y;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[0] = t > 0.0 ? 1.0 / sqrt(t) : 1.0;
    }
    __syncthreads();
    const double f = red[0];
    for (int g = threadIdx.x; g < ngw; g += blockDim.x) {
        x[g].x = (decltype(x[g].x))(x[g].x * f);
        x[g].y = (decltype(x[g].y))(x[g].y * f);
    }
}

int normalize_cols(Run &r, char *X, int ncols) {
    if (r.dtype == PW_C128)
        k_normalize_cols<double2><<<ncols, 256, 0, r.st>>>((double2 *)X, r.ldq, r.ngw);
    else
        k_normalize_cols<float2><<<ncols, 256, 0, r.st>>>((float2 *)X, r.ldq, r.ngw);
    CKR(r.c, cudaGetLastError());
    pwk_count_launches(r.c, 1);
    return PW_OK;
}

// T, G from the upper triangles of Hc, Sc; lowest nb pairs; eigenvectors
// (nbase x nb) into vc (ld nx), Ritz values into lam (device) and ew (host)
int reduced_eig(Run &r, const double2 *Hc, const double2 *Sc, int nx, int nbase, double2 *T, double2 *G, double2 *S,
                double2 *vc, double *lam, std::vector<double> &ew) {
    k_take_upper<<<blocks_for((size_t)nbase * nbase), 256, 0, r.st>>>(Hc, Sc, nx, T, G, nbase);
    CKR(r.c, cudaGetLastError());
    pwk_count_launches(r.c, 1);
    RK(eig(r, T, G, nbase, r.nb, lam, S));
    CKR(r.c, cudaMemcpy2DAsync(vc, nx * sizeof(double2), S, nbase * sizeof(double2), nbase * sizeof(double2), r.nb,
                               cudaMemcpyDeviceToDevice, r.st));
    CKR(r.c, cudaMemcpyAsync(ew.data(), lam, r.nb * sizeof(double), cudaMemcpyDeviceToHost, r.st));
    CKR(r.c, cudaStreamSynchronize(r.st));
    for (int i = 0; i < r.nb; ++i)
        if (!std::isfinite(ew[i])) return pwk_fail(r.c, PW_ERR_NAN, "non-finite Ritz value in Davidson");
    return PW_OK;
}

}  // namespace

extern "C" int pw_davidson(pw_ctx *c, int ik, int ispin, int dtype, void *X, int64_t ld, int nb, double tol,
                           int nitermax, double *evals, int *niter_out) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (!X || !evals || nb <= 0 || nitermax <= 0) return pwk_fail(c, PW_ERR_ARG, "bad pw_davidson arguments");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (ld < ngw || 2 * nb > ngw) return pwk_fail(c, PW_ERR_ARG, "bad pw_davidson shape (need ld >= Ngw and 2 nb <= Ngw)");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    r.dtype = dtype;
    r.es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    r.ngw = ngw;
    r.nb = nb;
    r.ldq = ngw;
    const int nx = 2 * nb;                              // Nvecx
    const size_t blk = (size_t)ngw * nb * r.es;
    char *psi, *Hpsi;
    RK(pwk_scratch(c, pwk::SL_LOB_Q, 2 * blk, (void **)&psi));
    RK(pwk_scratch(c, pwk::SL_LOB_HQ, 2 * blk, (void **)&Hpsi));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP1, blk, (void **)&r.T1));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP2, blk, (void **)&r.T2));
    const size_t s_xx = (size_t)nx * nx, s_xn = (size_t)nx * nb;
    // Hc, Sc, vc (nx x nx); T, G (nbase^2 <= nx^2); S, M, vc_prev (nx x nb);
    // lam, shifts (nx doubles each)
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, (5 * s_xx + 3 * s_xn + nx) * sizeof(double2), (void **)&r.small));
    r.eigw_bytes = pwk::eig_work_bytes(nx, nb);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    double2 *Hc = r.small, *Sc = Hc + s_xx, *vc = Sc + s_xx, *T = vc + s_xx, *G = T + s_xx;
    double2 *S = G + s_xx, *M = S + s_xn, *vc_prev = M + s_xn;
    double *lam = (double *)(vc_prev + s_xn), *shift = lam + nx;
    const bool mixed = dtype == PW_C64;
    auto col = [&](char *base, int j) { return base + (size_t)j * r.ldq * r.es; };

    // psi[:, 1:Nvec] = evc; Hpsi = H psi; Hc = psi'Hpsi, Sc = psi'psi (:67-72)
    CKR(c, cudaMemsetAsync(r.small, 0, 3 * s_xx * sizeof(double2), r.st));
    CKR(c, cudaMemcpy2DAsync(psi, r.ldq * r.es, X, ld * r.es, ngw * r.es, nb, cudaMemcpyDeviceToDevice, r.st));
    RK(pw_apply(c, ik, ispin, dtype, psi, Hpsi, r.ldq, nb, PW_OP_H));
    RK(gram_h(r, psi, nb, Hpsi, Hc, nx));
    RK(gram_h(r, psi, nb, psi, Sc, nx));
    std::vector<double> ew(nb), ev(nb), hshift(nb);
    std::vector<char> is_conv(nb, 0);
    RK(reduced_eig(r, Hc, Sc, nx, nb, T, G, S, vc, lam, ew));     // (:75-79)
    ev = ew;
    int nbase = nb, notcnv = nb, prev_nbase = nb, dav_iter = 0;
    bool have_evc = false;
    for (int kter = 1; kter <= nitermax; ++kter) {
        dav_iter = kter;
        // the last good Ritz coefficients, kept for the mixed-precision stop
        if (mixed) {
            CKR(c, cudaMemcpy2DAsync(vc_prev, nx * sizeof(double2), vc, nx * sizeof(double2), nbase * sizeof(double2),
                                     nb, cudaMemcpyDeviceToDevice, r.st));
            prev_nbase = nbase;
        }
        // unconverged roots first; their Ritz values are the shifts (:88-103)
        int np = 0;
        for (int ist = 0; ist < nb; ++ist) {
            if (is_conv[ist]) continue;
            if (np != ist)
                CKR(c, cudaMemcpyAsync(vc + (size_t)np * nx, vc + (size_t)ist * nx, nx * sizeof(double2),
                                       cudaMemcpyDeviceToDevice, r.st));
            hshift[np] = ev[ist];
            ++np;
        }
        // new vectors (H - e) psi vc, preconditioned, normalised (:107-127)
        char *pn = col(psi, nbase), *hn = col(Hpsi, nbase);
        CKR(c, cudaMemcpyAsync(shift, hshift.data(), notcnv * sizeof(double), cudaMemcpyHostToDevice, r.st));
        k_shift_cols<<<blocks_for((size_t)nbase * notcnv), 256, 0, r.st>>>(vc, nx, shift, M, nbase, notcnv);
        CKR(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        RK(rot(r, psi, nbase, M, nbase, notcnv, pn, 0));
        RK(rot(r, Hpsi, nbase, vc, nx, notcnv, pn, 1));
        RK(pw_kprec(c, ik, dtype, pn, pn, r.ldq, notcnv));
        RK(normalize_cols(r, pn, notcnv));
        // H psi_new; the new columns of the reduced matrices (:130-135)
        RK(pw_apply(c, ik, ispin, dtype, pn, hn, r.ldq, notcnv, PW_OP_H));
        RK(gram(r, psi, nbase + notcnv, hn, notcnv, Hc + (size_t)nbase * nx, nx));
        RK(gram(r, psi, nbase + notcnv, pn, notcnv, Sc + (size_t)nbase * nx, nx));
        nbase += notcnv;
        // diagonalise the reduced problem (:137-156)
        {
            const int s = reduced_eig(r, Hc, Sc, nx, nbase, T, G, S, vc, lam, ew);
            if (s == PW_ERR_NOT_POSDEF && mixed) {
                // the split-BF16 overlap lost definiteness: return the Ritz
                // vectors of the previous step
                ++r.restarts;
                RK(rot(r, psi, prev_nbase, vc_prev, nx, nb, r.T1, 0));
                have_evc = true;
                break;
            }
            RK(s);
        }
        // convergence test, new eigenvalues (:158-170)
        notcnv = 0;
        for (int i = 0; i < nb; ++i) {
            is_conv[i] = std::fabs(ew[i] - ev[i]) < tol;
            notcnv += !is_conv[i];
            ev[i] = ew[i];
        }
        // refresh the basis (:177-210)
        if (notcnv == 0 || nbase + notcnv > nx || kter == nitermax) {
            RK(rot(r, psi, nbase, vc, nx, nb, r.T1, 0));              // evc = psi vc
            have_evc = true;
            if (notcnv == 0 || kter == nitermax) break;
            RK(rot(r, Hpsi, nbase, vc, nx, nb, r.T2, 0));
            RK(copy_blk(r, psi, r.T1, nb));
            RK(copy_blk(r, Hpsi, r.T2, nb));
            nbase = nb;
            k_reset_reduced<<<blocks_for(s_xn), 256, 0, r.st>>>(Hc, Sc, vc, nx, nb, lam);
            CKR(c, cudaGetLastError());
            pwk_count_launches(c, 1);
        }
    }
    if (!have_evc) RK(rot(r, psi, nbase, vc, nx, nb, r.T1, 0));
    CKR(c, cudaMemcpy2DAsync(X, ld * r.es, r.T1, r.ldq * r.es, ngw * r.es, nb, cudaMemcpyDeviceToDevice, r.st));
    if (mixed) {
        k_normalize_cols<float2><<<nb, 256, 0, r.st>>>((float2 *)X, ld, ngw);
        CKR(c, cudaGetLastError());
        pwk_count_launches(c, 1);
    }
    CKR(c, cudaStreamSynchronize(r.st));
    for (int i = 0; i < nb; ++i) evals[i] = ev[i];
    if (niter_out) *niter_out = dav_iter + 1000 * r.restarts;
    return PW_OK;
}

// Host drop-in: X is the reference's host Matrix{ComplexF64} evc (Ngw x nb, ld).
extern "C" int pw_davidson_host(pw_ctx *c, int ik, int ispin, int dtype, double *X, int64_t ld, int nb, double tol,
                                int nitermax, double *evals, int *niter) {
    if (!c) return PW_ERR_ARG;
    if (!X || nb <= 0 || ld <= 0) return pwk_fail(c, PW_ERR_ARG, "bad pw_davidson_host arguments");
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    const size_t n = (size_t)ld * nb;
    void *d64 = nullptr, *d32 = nullptr;
    RK(pwk_scratch(c, pwk::SL_HOST_C128, n * sizeof(double2), &d64));
    CKR(c, cudaMemcpyAsync(d64, X, n * sizeof(double2), cudaMemcpyHostToDevice, st));
    void *dev = d64;
    if (dtype == PW_C64) {
        RK(pwk_scratch(c, pwk::SL_HOST_C64, n * sizeof(float2), &d32));
        CKR(c, pwk::convert_c128_to_c64((const double2 *)d64, (float2 *)d32, n, st));
        dev = d32;
    }
    RK(pw_davidson(c, ik, ispin, dtype, dev, ld, nb, tol, nitermax, evals, niter));
    if (dtype == PW_C64) CKR(c, pwk::convert_c64_to_c128((const float2 *)d32, (double2 *)d64, n, st));
    CKR(c, cudaMemcpyAsync(X, d64, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
    CKR(c, cudaStreamSynchronize(st));
    return PW_OK;
}
