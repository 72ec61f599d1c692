// pw_lobpcg: diag_LOBPCG! for one k-point (diag_LOBPCG.jl:51-225) with every
// block operation on the device: op_H and Kprec through pw_apply / pw_kprec,
// the Rayleigh-Ritz contractions through pw_gram / pw_rotate (tcgen05
// split-BF16x3 for complex64 blocks, FP64 CUDA cores for complex128), and the
// small FP64 Cholesky / eigen problems through the hand-written solver of
// pw_eig.cu.  The host only steers: it reads the nb eigenvalues per
// iteration for the convergence test (|evals - evals_old| < tol, as the
// reference).  The lock branch of the reference (devals <= 10 eps,
// :125-163) is not taken: its locking is replaced by the unlocked update.
// Mixed precision only: the reference's basis Q = [X W P] drifts towards
// linear dependence (lambda_min(Q'Q) ~ 1e-6 after a few iterations on Si64),
// which FP64 tolerates but a split-BF16 Gram (~1e-5 absolute error) does
// not; the mixed path therefore orthogonalises W against X and P, and the
// new P against the new X (block Gram-Schmidt, then Cholesky-QR as in the
// reference).  The Rayleigh-Ritz subspace span{X, W, P} of an iteration is
// unchanged by this; later iterates differ at round-off-amplified level and
// converge to the same Ritz values.  When the Cholesky of P'P fails the conjugate
// directions restart (P = W), and when that of W'W fails the iteration stops
// (residuals at the FP32 noise floor); the count of such events is returned
// as 1000 x restarts + iterations in *niter.  The FP64 path reports
// PW_ERR_NOT_POSDEF like the reference's cholesky.
#include <cmath>
#include <vector>

#include "pw_rr.cuh"


extern "C" int pw_eigh(pw_ctx *c, int n, int k, double *T, double *G, double *lam, double *S) {
    if (!c) return PW_ERR_ARG;
    if (n <= 0 || k <= 0 || k > n || !T || !lam) return pwk_fail(c, PW_ERR_ARG, "bad pw_eigh arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    r.eigw_bytes = pwk::eig_work_bytes(n, k);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    return eig(r, (double2 *)T, (double2 *)G, n, k, lam, (double2 *)S);
}

extern "C" int pw_lobpcg(pw_ctx *c, int ik, int ispin, int dtype, void *X, int64_t ld, int nb, double tol, int nitermax,
                         int nconv_target, double *evals, int *niter_out) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (!X || !evals || nb <= 0 || nitermax <= 0) return pwk_fail(c, PW_ERR_ARG, "bad pw_lobpcg arguments");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (ld < ngw || 3 * nb > ngw) return pwk_fail(c, PW_ERR_ARG, "bad pw_lobpcg shape (need ld >= Ngw and 3 nb <= Ngw)");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    if (nconv_target <= 0) nconv_target = nb;
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    r.dtype = dtype;
    r.es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    r.ngw = ngw;
    r.nb = nb;
    r.ldq = ngw;
    const size_t blk = (size_t)ngw * nb * r.es;
    RK(pwk_scratch(c, pwk::SL_LOB_Q, 3 * blk, (void **)&r.Q));
    RK(pwk_scratch(c, pwk::SL_LOB_HQ, 3 * blk, (void **)&r.HQ));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP1, 2 * blk, (void **)&r.T1));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP2, 2 * blk, (void **)&r.T2));
    const int n3 = 3 * nb;
    const size_t s_nn = (size_t)nb * nb, s_33 = (size_t)n3 * n3;
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, (4 * s_nn + 2 * s_33 + (size_t)n3 * nb + 2 * n3 + 8 * s_nn) * sizeof(double2),
                   (void **)&r.small));
    r.eigw_bytes = pwk::eig_work_bytes(n3, nb) > pwk::eig_work_bytes(nb, nb) ? pwk::eig_work_bytes(n3, nb)
                                                                             : pwk::eig_work_bytes(nb, nb);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    double2 *XHX = r.small, *M1 = XHX + s_nn, *Rinv = M1 + s_nn, *Sfin = Rinv + s_nn;
    double2 *T3 = Sfin + s_nn, *G3 = T3 + s_33, *S3 = G3 + s_33;
    double *lam = (double *)(S3 + (size_t)n3 * nb);
    double2 *T2b = (double2 *)(lam + 2 * (size_t)n3), *G2b = T2b + 4 * s_nn;   // [X W] blocks kept for a retry

    char *Xs = r.blk(r.Q, 0), *Ws = r.blk(r.Q, 1), *Ps = r.blk(r.Q, 2);
    char *HXs = r.blk(r.HQ, 0), *HWs = r.blk(r.HQ, 1), *HPs = r.blk(r.HQ, 2);
    // X -> Q[:, 0:nb]; HX = op_H(X)
    CKR(c, cudaMemcpy2DAsync(Xs, r.ldq * r.es, X, ld * r.es, ngw * r.es, nb, cudaMemcpyDeviceToDevice, r.st));
    RK(pw_apply(c, ik, ispin, dtype, Xs, HXs, r.ldq, nb, PW_OP_H));
    std::vector<double> ev(nb), ev_old(nb, 0.0);
    int it = 0;
    bool dropP = false;
    const double SMALL = 10.0 * 2.220446049250313e-16;
    (void)SMALL;
    for (it = 1; it <= nitermax; ++it) {
        // Rayleigh quotient XHX = X' HX and its eigenvalues (:85-86)
        RK(gram_h(r, Xs, nb, HXs, XHX, nb));
        k_herm_from_upper<<<blocks_for(s_nn), 256, 0, r.st>>>(XHX, nb);
        CKR(c, cudaMemcpyAsync(M1, XHX, s_nn * sizeof(double2), cudaMemcpyDeviceToDevice, r.st));
        RK(eig(r, M1, nullptr, nb, nb, lam, nullptr));
        CKR(c, cudaMemcpyAsync(ev.data(), lam, nb * sizeof(double), cudaMemcpyDeviceToHost, r.st));
        CKR(c, cudaStreamSynchronize(r.st));
        int nconv = 0;
        for (int i = 0; i < nb; ++i) {
            if (!std::isfinite(ev[i])) return pwk_fail(c, PW_ERR_NAN, "non-finite Ritz value in LOBPCG");
            if (std::fabs(ev[i] - ev_old[i]) < tol) ++nconv;
            ev_old[i] = ev[i];
        }
        if (nconv >= nconv_target) break;
        // R = HX - X XHX (:92), W = Kprec(R) (:123)
        RK(copy_blk(r, Ws, HXs, nb));
        k_scale_c128<<<blocks_for(s_nn), 256, 0, r.st>>>(XHX, M1, s_nn, -1.0);
        RK(rot(r, Xs, nb, M1, nb, nb, Ws, 1));
        RK(pw_kprec(c, ik, dtype, Ws, Ws, r.ldq, nb));
        // FP64 (reference order): HW = op_H(W); C = W'W = R^H R; W = W/R;
        // HW = HW/R (:167-174).
        // Mixed precision: keep Q = [X W P] near-orthonormal so that its
        // split-BF16 Gram stays positive definite (W -= X (X'W), W -= P (P'W),
        // twice is enough), normalise, and only then HW = op_H(W).  Carrying
        // HW through the projections and 1/R instead lets its FP32 rounding,
        // amplified by 1/R, drift away from H W; that drift reaches HX through
        // HQ U and grows every iteration.
        const bool mixed = dtype == PW_C64;
        if (!mixed) RK(pw_apply(c, ik, ispin, dtype, Ws, HWs, r.ldq, nb, PW_OP_H));
        if (mixed) {
            RK(project_out(r, Xs, nullptr, Ws, nullptr, M1));
            if (it > 1 && !dropP) {
                RK(project_out(r, Ps, nullptr, Ws, nullptr, M1));
                RK(project_out(r, Xs, nullptr, Ws, nullptr, M1));
            }
        }
        RK(gram_h(r, Ws, nb, Ws, M1, nb));
        {
            const int s = chol_rinv(r, M1, nb, Rinv);
            // mixed precision: a W'W that is not positive definite means the
            // residuals are at the noise floor of the FP32 blocks; stop here
            // (the FP64 path keeps the reference's behaviour and reports it)
            if (s == PW_ERR_NOT_POSDEF && dtype == PW_C64) {
                ++r.restarts;
                break;
            }
            RK(s);
        }
        RK(rot(r, Ws, nb, Rinv, nb, nb, r.T1, 0));
        RK(copy_blk(r, Ws, r.T1, nb));
        if (mixed) {
            RK(pw_apply(c, ik, ispin, dtype, Ws, HWs, r.ldq, nb, PW_OP_H));
        } else {
            RK(rot(r, HWs, nb, Rinv, nb, nb, r.T2, 0));
            RK(copy_blk(r, HWs, r.T2, nb));
        }
        // Rayleigh-Ritz on Q = [X W (P)] (:176-185)
        int nq = (it > 1 && !dropP) ? 3 * nb : 2 * nb;
        RK(gram_h(r, r.Q, nq, r.HQ, T3, nq));
        RK(gram_h(r, r.Q, nq, r.Q, G3, nq));
        if (dtype == PW_C64 && nq == 3 * nb) {
            const size_t w2 = 2 * (size_t)nb * sizeof(double2);
            CKR(c, cudaMemcpy2DAsync(T2b, w2, T3, nq * sizeof(double2), w2, 2 * nb, cudaMemcpyDeviceToDevice, r.st));
            CKR(c, cudaMemcpy2DAsync(G2b, w2, G3, nq * sizeof(double2), w2, 2 * nb, cudaMemcpyDeviceToDevice, r.st));
        }
        {
            int s = eig(r, T3, G3, nq, nb, lam, S3);
            if (s == PW_ERR_NOT_POSDEF && dtype == PW_C64 && nq == 3 * nb) {
                // mixed precision: Q'Q lost definiteness through P; redo the
                // Rayleigh-Ritz on [X W] and restart P = W (as iteration 1)
                ++r.restarts;
                nq = 2 * nb;
                s = eig(r, T2b, G2b, nq, nb, lam, S3);
            }
            if (s == PW_ERR_NOT_POSDEF && dtype == PW_C64) {
                // [X W] itself is not definite: W is at the FP32 noise floor,
                // the block has converged as far as this precision allows
                ++r.restarts;
                break;
            }
            RK(s);
        }
        const bool usedP = (nq == 3 * nb);
        // X = Q U, HX = HQ U  (:187-189) into the temporaries
        RK(rot(r, r.Q, nq, S3, nq, nb, r.T1, 0));
        RK(rot(r, r.HQ, nq, S3, nq, nb, r.T2, 0));
        if (usedP) {
            // P = [W P] U[nb:3nb], HP = [HW HP] U[nb:3nb]; P = P/R, HP = HP/R (:190-199)
            char *Pn = r.T1 + blk, *HPn = r.T2 + blk;
            RK(rot(r, Ws, 2 * nb, S3 + nb, nq, nb, Pn, 0));
            RK(rot(r, HWs, 2 * nb, S3 + nb, nq, nb, HPn, 0));
            if (dtype == PW_C64) RK(project_out(r, r.T1, r.T2, Pn, HPn, M1));   // P -= Xnew (Xnew'P)
            RK(gram_h(r, Pn, nb, Pn, M1, nb));
            const int s = chol_rinv(r, M1, nb, Rinv);
            if (s == PW_ERR_NOT_POSDEF && dtype == PW_C64) {
                // mixed precision: restart the conjugate directions, P = W
                ++r.restarts;
                RK(copy_blk(r, Ps, Ws, nb));
                RK(copy_blk(r, HPs, HWs, nb));
            } else {
                RK(s);
                RK(rot(r, Pn, nb, Rinv, nb, nb, Ps, 0));
                RK(rot(r, HPn, nb, Rinv, nb, nb, HPs, 0));
            }
        } else {
            // P = W, HP = HW (:201-202)
            RK(copy_blk(r, Ps, Ws, nb));
            RK(copy_blk(r, HPs, HWs, nb));
        }
        RK(copy_blk(r, Xs, r.T1, nb));
        RK(copy_blk(r, HXs, r.T2, nb));
        dropP = false;
    }
    if (it > nitermax) it = nitermax;
    // final Rayleigh-Ritz: S = X'HX, S = (S+S')/2, X = X Q (:214-217)
    RK(gram(r, Xs, nb, HXs, nb, Sfin, nb));
    k_herm_avg<<<blocks_for(s_nn), 256, 0, r.st>>>(Sfin, nb);
    RK(eig(r, Sfin, nullptr, nb, nb, lam, M1));
    RK(rot(r, Xs, nb, M1, nb, nb, r.T1, 0));
    CKR(c, cudaMemcpy2DAsync(X, ld * r.es, r.T1, r.ldq * r.es, ngw * r.es, nb, cudaMemcpyDeviceToDevice, r.st));
    if (dtype == PW_C64) {
        k_normalize_cols_c64<<<nb, 256, 0, r.st>>>((float2 *)X, ld, ngw);
        CKR(c, cudaGetLastError());
    }
    CKR(c, cudaMemcpyAsync(evals, lam, nb * sizeof(double), cudaMemcpyDeviceToHost, r.st));
    CKR(c, cudaStreamSynchronize(r.st));
    if (niter_out) *niter_out = it + 1000 * r.restarts;
    return PW_OK;
}

// Host drop-in: X is the reference's host Matrix{ComplexF64} (Ngw x nb, ld).
extern "C" int pw_lobpcg_host(pw_ctx *c, int ik, int ispin, int dtype, double *X, int64_t ld, int nb, double tol,
                              int nitermax, int nconv, double *evals, int *niter) {
    if (!c) return PW_ERR_ARG;
    if (!X || nb <= 0 || ld <= 0) return pwk_fail(c, PW_ERR_ARG, "bad pw_lobpcg_host arguments");
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
    RK(pw_lobpcg(c, ik, ispin, dtype, dev, ld, nb, tol, nitermax, nconv, evals, niter));
    if (dtype == PW_C64) CKR(c, pwk::convert_c64_to_c128((const float2 *)d32, (double2 *)d64, n, st));
    CKR(c, cudaMemcpyAsync(X, d64, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
    CKR(c, cudaStreamSynchronize(st));
    return PW_OK;
}

// ortho_sqrt! (ortho_sqrt.jl:1-11): psi := psi * inv(sqrt(psi'psi)), with
// psi'psi = U diag(lam) U^H from the FP64 eigensolver and
// inv(sqrt(.)) = U diag(lam^-1/2) U^H.
namespace {
__global__ void k_scale_cols(const double2 *U, const double *lam, double2 *V, int n) {
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n);
        const double s = 1.0 / sqrt(lam[j]);
        V[t] = make_double2(U[t].x * s, U[t].y * s);
    }
}
}  // namespace

extern "C" int pw_ortho_sqrt(pw_ctx *c, int dtype, void *psi, int64_t ld, int64_t ngw, int nb) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (!psi || nb <= 0 || ngw <= 0 || ld < ngw) return pwk_fail(c, PW_ERR_ARG, "bad pw_ortho_sqrt arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    const size_t es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    const size_t nn = (size_t)nb * nb;
    double2 *S = nullptr, *U = nullptr, *M = nullptr, *V = nullptr;
    double *lam = nullptr;
    char *tmp = nullptr;
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, 4 * nn * sizeof(double2) + nb * sizeof(double) + 256, (void **)&S));
    U = S + nn;
    V = U + nn;
    M = V + nn;
    lam = (double *)(M + nn);
    RK(pwk_scratch(c, pwk::SL_LOB_TMP1, (size_t)ld * nb * es, (void **)&tmp));
    r.eigw_bytes = pwk::eig_work_bytes(nb, nb);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    RK(pw_gram(c, dtype, ngw, nb, nb, psi, ld, psi, ld, (double *)S, nb, 0));
    RK(eig(r, S, nullptr, nb, nb, lam, U));
    std::vector<double> hl(nb);
    CKR(c, cudaMemcpyAsync(hl.data(), lam, nb * sizeof(double), cudaMemcpyDeviceToHost, r.st));
    CKR(c, cudaStreamSynchronize(r.st));
    for (double x : hl)
        if (!(x > 0.0)) return pwk_fail(c, PW_ERR_NOT_POSDEF, "psi'psi is not positive definite");
    k_scale_cols<<<blocks_for(nn), 256, 0, r.st>>>(U, lam, V, nb);
    // M = (U diag(lam^-1/2)) U^H : the C128 rotate computes A * W with A = V (n x n)
    // and W = U^H (conj-transposed on the host side of this call)
    std::vector<double2> hu(nn), huh(nn);
    CKR(c, cudaMemcpyAsync(hu.data(), U, nn * sizeof(double2), cudaMemcpyDeviceToHost, r.st));
    CKR(c, cudaStreamSynchronize(r.st));
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) huh[(size_t)j * nb + i] = make_double2(hu[(size_t)i * nb + j].x, -hu[(size_t)i * nb + j].y);
    CKR(c, cudaMemcpyAsync(S, huh.data(), nn * sizeof(double2), cudaMemcpyHostToDevice, r.st));
    RK(pw_rotate(c, PW_C128, nb, nb, nb, V, nb, (const double *)S, nb, M, nb, 0));
    RK(pw_rotate(c, dtype, ngw, nb, nb, psi, ld, (const double *)M, nb, tmp, ld, 0));
    CKR(c, cudaMemcpy2DAsync(psi, ld * es, tmp, ld * es, ngw * es, nb, cudaMemcpyDeviceToDevice, r.st));
    CKR(c, cudaStreamSynchronize(r.st));
    return PW_OK;
}

// Rinv = inv(cholesky(Hermitian(C)).U) (the W / R and P / R of
// diag_LOBPCG.jl:144-147,170-174,195-199), C read from its upper triangle and
// overwritten; FP64 on the device.
extern "C" int pw_chol_rinv(pw_ctx *c, int n, double *C, double *Rinv) {
    if (!c) return PW_ERR_ARG;
    if (!C || !Rinv || n <= 0 || C == Rinv) return pwk_fail(c, PW_ERR_ARG, "bad pw_chol_rinv arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    r.eigw_bytes = pwk::eig_work_bytes(n, 1);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    return chol_rinv(r, (double2 *)C, n, (double2 *)Rinv);
}

// ortho_cholesky!(psi) (ortho_sqrt.jl:80-89): O = psi'psi = U^H U (Cholesky),
// psi := psi / U.
extern "C" int pw_ortho_cholesky(pw_ctx *c, int dtype, void *psi, int64_t ld, int64_t ngw, int nb) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (!psi || nb <= 0 || ngw <= 0 || ld < ngw) return pwk_fail(c, PW_ERR_ARG, "bad pw_ortho_cholesky arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    Run r{};
    r.c = c;
    r.st = pwk_stream(c);
    r.dtype = dtype;
    r.ngw = (int)ngw;
    r.ldq = ld;
    r.nb = nb;
    const size_t es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    const size_t nn = (size_t)nb * nb;
    double2 *O = nullptr, *Rinv = nullptr;
    char *tmp = nullptr;
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, 2 * nn * sizeof(double2) + 256, (void **)&O));
    Rinv = O + nn;
    RK(pwk_scratch(c, pwk::SL_LOB_TMP1, (size_t)ld * nb * es, (void **)&tmp));
    r.eigw_bytes = pwk::eig_work_bytes(nb, 1);
    RK(pwk_scratch(c, pwk::SL_LOB_EIGW, r.eigw_bytes, &r.eigw));
    RK(pwk_scratch(c, pwk::SL_LOB_EIGSTAT, 64, (void **)&r.eigstat));
    RK(gram_h(r, (const char *)psi, nb, (const char *)psi, O, nb));
    RK(chol_rinv(r, O, nb, Rinv));
    RK(pw_rotate(c, dtype, ngw, nb, nb, psi, ld, (const double *)Rinv, nb, tmp, ld, 0));
    CKR(c, cudaMemcpy2DAsync(psi, ld * es, tmp, ld * es, ngw * es, nb, cudaMemcpyDeviceToDevice, r.st));
    CKR(c, cudaStreamSynchronize(r.st));
    return PW_OK;
}

// calc_grad (calc_grad.jl:1-57): grad_i = wk f_i (H psi_i - sum_j psi_j <psi_j|H psi_i>),
// plus psi Q with Q = (Hred F - F Hred)/2 when the occupations are not all
// equal to 2 or all equal to 1 (Hred = psi'H psi, F = diag(f)).
// As matrices: grad = (H psi) D + psi (-Hred D + Q), D = wk F.
namespace {
__global__ void k_grad_coef(const double2 *__restrict__ Hm, const double *__restrict__ f, double wk, int nb, int frac,
                            double2 *__restrict__ U) {
    const size_t total = (size_t)nb * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / nb), i = (int)(t - (size_t)j * nb);
        const double2 h = Hm[t];
        double s = -wk * f[j];
        if (frac) s += 0.5 * (f[j] - f[i]);
        U[t] = make_double2(h.x * s, h.y * s);
    }
}
template <typename T>
__global__ void k_scale_cols_w(Cx<T> *__restrict__ X, int64_t ld, int ngw, int nb, const double *__restrict__ f, double wk) {
    const size_t total = (size_t)ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / ngw), g = (int)(t - (size_t)b * ngw);
        const T s = (T)(wk * f[b]);
        Cx<T> &x = X[(size_t)b * ld + g];
        x = cmake(x.x * s, x.y * s);
    }
}
}  // namespace

extern "C" int pw_calc_grad(pw_ctx *c, int ik, int ispin, int dtype, const void *psi, void *grad, int64_t ld, int nb,
                            const double *Focc, double wk) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (!psi || !grad || !Focc || nb <= 0 || ld < ngw || psi == grad) return pwk_fail(c, PW_ERR_ARG, "bad pw_calc_grad arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    bool all2 = true, all1 = true;
    for (int i = 0; i < nb; ++i) {
        all2 = all2 && Focc[i] == 2.0;
        all1 = all1 && Focc[i] == 1.0;
    }
    const int frac = (all2 || all1) ? 0 : 1;
    const size_t nn = (size_t)nb * nb;
    double2 *Hm = nullptr, *U = nullptr;
    double *df = nullptr;
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, 2 * nn * sizeof(double2) + (size_t)nb * sizeof(double) + 256, (void **)&Hm));
    U = Hm + nn;
    df = (double *)(U + nn);
    CKR(c, cudaMemcpyAsync(df, Focc, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, st));
    RK(pw_apply(c, ik, ispin, dtype, psi, grad, ld, nb, PW_OP_H));
    RK(pw_gram(c, dtype, ngw, nb, nb, psi, ld, grad, ld, (double *)Hm, nb, 0));
    k_grad_coef<<<blocks_for(nn), 256, 0, st>>>(Hm, df, wk, nb, frac, U);
    const int nblk = blocks_for((size_t)ngw * nb);
    if (dtype == PW_C128)
        k_scale_cols_w<double><<<nblk, 256, 0, st>>>((double2 *)grad, ld, ngw, nb, df, wk);
    else
        k_scale_cols_w<float><<<nblk, 256, 0, st>>>((float2 *)grad, ld, ngw, nb, df, wk);
    CKR(c, cudaGetLastError());
    RK(pw_rotate(c, dtype, ngw, nb, nb, psi, ld, (const double *)U, nb, grad, ld, 1));
    pwk_count_launches(c, 2);
    return PW_OK;
}
