// The device parts of diag_CheFSI! (CheFSI.jl:1-139):
//   pw_chebyfilt       chebyfilt (CheFSI.jl:34-64): the scaled Chebyshev filter
//                      of degree m applied to a block, m op_H applications and
//                      one fused three-term combination kernel per step;
//   pw_lanczos_bounds  get_ub_lb_lanczos (CheFSI.jl:67-125) with
//                      norm_matrix_induced (CheFSI.jl:128-138): nlancz Lanczos
//                      steps with one step of full reorthogonalisation, in
//                      FP64, the Lanczos vectors kept on the device.
// The ortho_sqrt! and the Rayleigh quotient of diag_CheFSI! are pw_ortho_sqrt,
// pw_apply, pw_gram and pw_eigh; the host wrapper (pwb200/chefsi.py) strings
// them together per k-point as the reference does.
#include <vector>

#include "pw_rr.cuh"

namespace {

// out = a HY + b Y + d X (X null: d ignored) over nb rows of ngw (stride
// ld).  out may be X itself: each element is read before it is written by
// the same thread.
template <typename C>
__global__ void k_cheb_comb(const C *HY, const C *Y, const C *X, C *out, int64_t ld, int ngw, int nb, double a,
                            double b, double d) {
    using R = decltype(HY->x);
    const R ra = (R)a, rb = (R)b, rd = (R)d;
    const size_t total = (size_t)ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t j = t / ngw, g = t - j * ngw, o = j * ld + g;
        const C h = HY[o], y = Y[o];
        R re = ra * h.x + rb * y.x, im = ra * h.y + rb * y.y;
        if (X) {
            const C x = X[o];
            re += rd * x.x;
            im += rd * x.y;
        }
        C r;
        r.x = re;
        r.y = im;
        out[o] = r;
    }
}

int cheb_comb(pw_ctx *c, int dtype, const void *HY, const void *Y, const void *X, void *out, int64_t ld, int ngw,
              int nb, double a, double b, double d, cudaStream_t st) {
    const int grid = blocks_for((size_t)ngw * nb);
    if (dtype == PW_C128)
        k_cheb_comb<double2><<<grid, 256, 0, st>>>((const double2 *)HY, (const double2 *)Y, (const double2 *)X,
                                                    (double2 *)out, ld, ngw, nb, a, b, d);
    else
        k_cheb_comb<float2><<<grid, 256, 0, st>>>((const float2 *)HY, (const float2 *)Y, (const float2 *)X,
                                                   (float2 *)out, ld, ngw, nb, a, b, d);
    CKR(c, cudaGetLastError());
    pwk_count_launches(c, 1);
    return PW_OK;
}

// s = ||f|| in FP64 (one CTA); vj = f / s when vj is given; T[j, j-1] = s
// (column-major, order n) when T is given and j > 0; *sout = s when given.
__global__ void k_lz_norm(const double2 *f, int ngw, double2 *vj, double *T, int n, int j, double *sout) {
    __shared__ double red[32];
    double s = 0.0;
    for (int g = threadIdx.x; g < ngw; g += blockDim.x) s += f[g].x * f[g].x + f[g].y * f[g].y;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[0] = sqrt(t);
    }
    __syncthreads();
    const double nrm = red[0];
    if (vj)
        for (int g = threadIdx.x; g < ngw; g += blockDim.x) vj[g] = make_double2(f[g].x / nrm, f[g].y / nrm);
    if (threadIdx.x == 0) {
        if (T && j > 0) T[(size_t)(j - 1) * n + j] = nrm;
        if (sout) *sout = nrm;
    }
}

// first step (CheFSI.jl:87-95): h1 = Re(V1' HV1) is both T[1,1] and the
// coefficient subtracted before the reorthogonalisation: nh = -h1
__global__ void k_lz_first(const double2 *h, double *T, double2 *nh) {
    T[0] = h[0].x;
    nh[0] = make_double2(-h[0].x, 0.0);
}
// nh = -h (m entries)
__global__ void k_lz_neg(const double2 *h, double2 *nh, int m) {
    for (int i = threadIdx.x; i < m; i += blockDim.x) nh[i] = make_double2(-h[i].x, -h[i].y);
}
// reorthogonalisation bookkeeping of step j (CheFSI.jl:108-114): h += s,
// T[1:m, j] = Re h, nh = -s
__global__ void k_lz_fin(double2 *h, const double2 *s, double *T, int n, int j, int m, double2 *nh) {
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double2 v = make_double2(h[i].x + s[i].x, h[i].y + s[i].y);
        h[i] = v;
        T[(size_t)j * n + i] = v.x;
        nh[i] = make_double2(-s[i].x, -s[i].y);
    }
}
// complex copy of a real n x n matrix (the eigensolver reads the upper triangle)
__global__ void k_real_to_c(const double *T, double2 *Tc, size_t nn) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nn; t += (size_t)gridDim.x * blockDim.x)
        Tc[t] = make_double2(T[t], 0.0);
}

}  // namespace

extern "C" int pw_chebyfilt(pw_ctx *c, int ik, int ispin, int dtype, const void *X, void *Y, int64_t ld, int nb,
                            int degree, double lb, double ub) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (!X || !Y || X == Y || nb <= 0 || degree < 1) return pwk_fail(c, PW_ERR_ARG, "bad pw_chebyfilt arguments");
    if (!(ub > lb) || !std::isfinite(lb) || !std::isfinite(ub))
        return pwk_fail(c, PW_ERR_ARG, "pw_chebyfilt needs finite bounds with ub > lb");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (ld < ngw) return pwk_fail(c, PW_ERR_ARG, "ld < Ngw");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    const size_t es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    const size_t blk = (size_t)ld * nb * es;
    char *B1, *HY;
    RK(pwk_scratch(c, pwk::SL_LOB_Q, blk, (void **)&B1));
    RK(pwk_scratch(c, pwk::SL_LOB_HQ, blk, (void **)&HY));
    // CheFSI.jl:48-53: half width e, centre c, sigma = e / (lb - ub), sigma1 fixed
    const double e = 0.5 * (ub - lb), cc = 0.5 * (ub + lb), sigma1 = e / (lb - ub);
    double sigma = sigma1;
    // iterate i (1-based) lives in Y when degree - i is even, else in B1, so
    // the last one lands in Y and iterate i overwrites iterate i - 2 in place
    auto buf = [&](int i) { return ((degree - i) % 2 == 0) ? (char *)Y : B1; };
    // Y = (H X - c X) sigma1 / e (CheFSI.jl:58-59)
    RK(pw_apply(c, ik, ispin, dtype, X, HY, ld, nb, PW_OP_H));
    RK(cheb_comb(c, dtype, HY, X, nullptr, buf(1), ld, ngw, nb, sigma1 / e, -cc * sigma1 / e, 0.0, st));
    const void *prev = X;
    for (int i = 2; i <= degree; ++i) {
        // sigma2 = 1 / (2 / sigma1 - sigma); Y1 = (H Y - c Y) 2 sigma2 / e - X sigma sigma2 (CheFSI.jl:61-66)
        const double sigma2 = 1.0 / (2.0 / sigma1 - sigma);
        char *cur = buf(i - 1), *nxt = buf(i);
        RK(pw_apply(c, ik, ispin, dtype, cur, HY, ld, nb, PW_OP_H));
        RK(cheb_comb(c, dtype, HY, cur, prev, nxt, ld, ngw, nb, 2.0 * sigma2 / e, -2.0 * cc * sigma2 / e,
                     -sigma * sigma2, st));
        prev = cur;
        sigma = sigma2;
    }
    return PW_OK;
}

extern "C" int pw_lanczos_bounds(pw_ctx *c, int ik, int ispin, int nlancz, const double *v0, double *lb, double *ub) {
    if (!c) return PW_ERR_ARG;
    if (!v0 || !lb || !ub || nlancz < 2 || nlancz % 2) return pwk_fail(c, PW_ERR_ARG, "bad pw_lanczos_bounds arguments (nlancz even >= 2)");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (nlancz > ngw) return pwk_fail(c, PW_ERR_ARG, "nlancz > Ngw");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    const int n = nlancz;
    const size_t vb = (size_t)ngw * sizeof(double2);
    double2 *V, *HV, *small, *Tc;
    double *lam;
    RK(pwk_scratch(c, pwk::SL_LOB_Q, (size_t)n * vb, (void **)&V));
    RK(pwk_scratch(c, pwk::SL_LOB_HQ, 2 * vb, (void **)&HV));
    // h, s, nh (n each), then T (n x n real) and ||f||
    RK(pwk_scratch(c, pwk::SL_LOB_SMALL, 3 * (size_t)n * sizeof(double2) + ((size_t)n * n + 1) * sizeof(double),
                   (void **)&small));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP1, (size_t)n * n * sizeof(double2), (void **)&Tc));
    RK(pwk_scratch(c, pwk::SL_LOB_TMP2, (size_t)n * sizeof(double), (void **)&lam));
    double2 *f = HV + ngw, *h = small, *s = h + n, *nh = s + n;
    double *T = (double *)(nh + n), *fnorm = T + (size_t)n * n;
    CKR(c, cudaMemsetAsync(T, 0, (size_t)n * n * sizeof(double), st));
    auto Vc = [&](int j) { return (const void *)(V + (size_t)j * ngw); };
    // V1 = v0 / ||v0||; HV1 = H V1; h1 = Re(V1' HV1) = T[1,1]; f = HV1 - V1 h1;
    // s1 = V1' f; f -= V1 s1 (CheFSI.jl:84-95)
    k_lz_norm<<<1, 1024, 0, st>>>((const double2 *)v0, ngw, V, nullptr, n, 0, nullptr);
    CKR(c, cudaGetLastError());
    RK(pw_apply(c, ik, ispin, PW_C128, Vc(0), HV, ngw, 1, PW_OP_H));
    RK(pw_gram(c, PW_C128, ngw, 1, 1, Vc(0), ngw, HV, ngw, (double *)h, 1, 0));
    k_lz_first<<<1, 1, 0, st>>>(h, T, nh);
    CKR(c, cudaGetLastError());
    CKR(c, cudaMemcpyAsync(f, HV, vb, cudaMemcpyDeviceToDevice, st));
    RK(pw_rotate(c, PW_C128, ngw, 1, 1, Vc(0), ngw, (const double *)nh, 1, f, ngw, 1));
    RK(pw_gram(c, PW_C128, ngw, 1, 1, Vc(0), ngw, f, ngw, (double *)s, 1, 0));
    k_lz_neg<<<1, 32, 0, st>>>(s, nh, 1);
    CKR(c, cudaGetLastError());
    RK(pw_rotate(c, PW_C128, ngw, 1, 1, Vc(0), ngw, (const double *)nh, 1, f, ngw, 1));
    pwk_count_launches(c, 3);
    for (int j = 1; j < n; ++j) {
        const int m = j + 1;
        // beta = ||f||, T[j, j-1] = beta, V_j = f / beta, HV_j = H V_j (:98-102)
        k_lz_norm<<<1, 1024, 0, st>>>(f, ngw, V + (size_t)j * ngw, T, n, j, nullptr);
        CKR(c, cudaGetLastError());
        RK(pw_apply(c, ik, ispin, PW_C128, Vc(j), HV, ngw, 1, PW_OP_H));
        // h = V[:, 1:j]' HV_j; f = HV_j - V h (:104-107)
        RK(pw_gram(c, PW_C128, ngw, m, 1, V, ngw, HV, ngw, (double *)h, m, 0));
        k_lz_neg<<<1, 256, 0, st>>>(h, nh, m);
        CKR(c, cudaGetLastError());
        CKR(c, cudaMemcpyAsync(f, HV, vb, cudaMemcpyDeviceToDevice, st));
        RK(pw_rotate(c, PW_C128, ngw, 1, m, V, ngw, (const double *)nh, m, f, ngw, 1));
        // s = V' f; h += s; f -= V s; T[1:j, j] = Re h (:109-118)
        RK(pw_gram(c, PW_C128, ngw, m, 1, V, ngw, f, ngw, (double *)s, m, 0));
        k_lz_fin<<<1, 256, 0, st>>>(h, s, T, n, j, m, nh);
        CKR(c, cudaGetLastError());
        RK(pw_rotate(c, PW_C128, ngw, 1, m, V, ngw, (const double *)nh, m, f, ngw, 1));
        pwk_count_launches(c, 3);
    }
    k_lz_norm<<<1, 1024, 0, st>>>(f, ngw, nullptr, nullptr, n, 0, fnorm);
    CKR(c, cudaGetLastError());
    std::vector<double> Th((size_t)n * n + 1);
    CKR(c, cudaMemcpyAsync(Th.data(), T, Th.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKR(c, cudaStreamSynchronize(st));
    for (double v : Th)
        if (!std::isfinite(v)) return pwk_fail(c, PW_ERR_NAN, "non-finite Lanczos coefficient (breakdown)");
    // ub = norm_matrix_induced(T) + ||f|| = ||T 1/sqrt(n)|| + ||f|| (:121, :127-137)
    double nrm2 = 0.0;
    const double d = 1.0 / std::sqrt((double)n);
    for (int i = 0; i < n; ++i) {
        double r = 0.0;
        for (int j = 0; j < n; ++j) r += Th[(size_t)j * n + i] * d;
        nrm2 += r * r;
    }
    *ub = std::sqrt(nrm2) + Th[(size_t)n * n];
    // lb = eigvals(T)[nlancz / 2] (:119-120).  T is the Lanczos matrix:
    // its upper triangle holds the reorthogonalised coefficients and its
    // subdiagonal the betas, equal to the superdiagonal to rounding, so the
    // Hermitian solver on the upper triangle stands in for the reference's
    // general eigvals.
    k_real_to_c<<<blocks_for((size_t)n * n), 256, 0, st>>>(T, Tc, (size_t)n * n);
    CKR(c, cudaGetLastError());
    pwk_count_launches(c, 2);
    RK(pw_eigh(c, n, n / 2, (double *)Tc, nullptr, lam, nullptr));
    CKR(c, cudaMemcpyAsync(lb, lam + (n / 2 - 1), sizeof(double), cudaMemcpyDeviceToHost, st));
    CKR(c, cudaStreamSynchronize(st));
    return PW_OK;
}
