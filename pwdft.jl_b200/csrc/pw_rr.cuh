// Shared helpers of the device eigensolvers (pw_lobpcg.cu, pw_davidson.cu):
// the per-call state (block storage, small FP64 matrices, eigensolver
// workspace), the small FP64 eigen/Cholesky steps and the block products
// through pw_gram / pw_rotate.  Included by one translation unit each;
// everything lives in an unnamed namespace.
#pragma once
#include <cmath>
#include <cstring>

#include "../../include/pwb200.h"
#include "pw_eig.h"
#include "pw_launch.h"

int pwk_fail(pw_ctx *c, int code, const char *msg);
int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out);
int pwk_gram_upper(pw_ctx *c, int dtype, int64_t K, int m, const void *A, int64_t lda, const void *B, int64_t ldb,
                   double *C, int64_t ldc);
cudaStream_t pwk_stream(pw_ctx *c);
int pwk_ngw(const pw_ctx *c, int ik);
int pwk_device(const pw_ctx *c);
int pwk_nkpt(const pw_ctx *c);
void pwk_count_launches(pw_ctx *c, int n);

namespace {


__global__ void k_scale_c128(const double2 *in, double2 *out, size_t n, double s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_double2(in[i].x * s, in[i].y * s);
}
// S := (S + S^H)/2 written to both triangles
__global__ void k_herm_avg(double2 *S, int n) {
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        if (i < j) {
            const double2 a = S[t], b = S[(size_t)i * n + j];
            const double2 m = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            S[t] = m;
            S[(size_t)i * n + j] = make_double2(m.x, -m.y);
        } else if (i == j) {
            S[t].y = 0.0;
        }
    }
}
// lower := conj(upper)^T (Julia's Hermitian(A)), diagonal made real
__global__ void k_herm_from_upper(double2 *A, int n) {
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        if (i > j) {
            const double2 u = A[(size_t)i * n + j];
            A[t] = make_double2(u.x, -u.y);
        } else if (i == j) {
            A[t].y = 0.0;
        }
    }
}
int blocks_for(size_t total) {
    size_t b = (total + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return b < 1 ? 1 : (int)b;
}

struct Run {
    pw_ctx *c;
    cudaStream_t st;
    int dtype;
    size_t es;
    int ngw, nb;
    int64_t ldq;
    char *Q, *HQ, *T1, *T2;     // Q = [X W P], HQ = [HX HW HP], two Ngw x 2nb temporaries
    double2 *small;             // small FP64 complex matrices
    void *eigw;
    size_t eigw_bytes;
    int *eigstat;
    int restarts = 0;           // mixed-precision safeguards taken (see pw_lobpcg)

    char *blk(char *base, int j) const { return base + (size_t)j * nb * ldq * es; }
};

#define RK(x)                     \
    do {                          \
        int s_ = (x);             \
        if (s_ != PW_OK) return s_; \
    } while (0)
#define CKR(c, x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, #x " failed"); \
    } while (0)

// lowest k eigenpairs of (T, G) (G may be null) of order n; T, G overwritten
int eig(Run &r, double2 *T, double2 *G, int n, int k, double *lam_dev, double2 *S) {
    CKR(r.c, pwk::hegv_lowest(T, G, n, k, lam_dev, S, r.eigw, r.eigw_bytes, nullptr, r.eigstat, r.st));
    int h[3] = {0, 0, 0};
    CKR(r.c, cudaMemcpyAsync(h, r.eigstat, sizeof(h), cudaMemcpyDeviceToHost, r.st));
    CKR(r.c, cudaStreamSynchronize(r.st));
    if (h[0]) return pwk_fail(r.c, PW_ERR_TIMEOUT, "a bounded grid barrier of the eigensolver expired");
    if (h[1]) return pwk_fail(r.c, PW_ERR_NOT_POSDEF, "overlap matrix not positive definite (Cholesky)");
    if (h[2]) return pwk_fail(r.c, PW_ERR_NAN, "non-finite value in the eigenproblem");
    pwk_count_launches(r.c, 10);
    return PW_OK;
}

// upper Cholesky factor R of the Hermitian C (C = R^H R) and Rinv = R^-1:
// via the generalized solver with T = I would cost too much, so use the
// lower factor of pw_eig's Cholesky: returns Rinv in `Rinv` (n x n).
int chol_rinv(Run &r, double2 *C, int n, double2 *Rinv);

// X (Ngw x k block, ld ldq) := X * M  (M: k x n device FP64 complex, ld ldm) into out
int rot(Run &r, const char *A, int k, const double2 *M, int ldm, int n, char *out, int acc) {
    return pw_rotate(r.c, r.dtype, r.ngw, n, k, A, r.ldq, (const double *)M, ldm, out, r.ldq, acc);
}
int gram(Run &r, const char *A, int m, const char *B, int n, double2 *C, int ldc) {
    return pw_gram(r.c, r.dtype, r.ngw, m, n, A, r.ldq, B, r.ldq, (double *)C, ldc, 0);
}
// Hermitian products (X'HX, Q'HQ, Q'Q, W'W, P'P): upper triangle only, which
// is all their consumers read
int gram_h(Run &r, const char *A, int m, const char *B, double2 *C, int ldc) {
    return pwk_gram_upper(r.c, r.dtype, r.ngw, m, A, r.ldq, B, r.ldq, (double *)C, ldc);
}
int copy_blk(Run &r, char *dst, const char *src, int ncols) {
    CKR(r.c, cudaMemcpy2DAsync(dst, r.ldq * r.es, src, r.ldq * r.es, r.ngw * r.es, ncols, cudaMemcpyDeviceToDevice, r.st));
    return PW_OK;
}

// B -= A (A'B) and HB -= HA (A'B) for nb-column blocks (A orthonormal):
// the block Gram-Schmidt step of the mixed-precision LOBPCG.  M: nb x nb scratch.
// Mixed precision: each column of the FP32 block rescaled to unit norm,
// the norm summed in FP64 (one CTA per column).  The split-BF16 Gram keeps
// X orthonormal to about 1e-5; this makes the norms, and so the electron
// count of calc_rhoe, exact to FP32 rounding.
__global__ void k_normalize_cols_c64(float2 *X, int64_t ld, int ngw) {
    __shared__ double red[32];
    float2 *x = X + (size_t)blockIdx.x * ld;
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
    const float f = (float)red[0];
    for (int g = threadIdx.x; g < ngw; g += blockDim.x) x[g] = make_float2(x[g].x * f, x[g].y * f);
}

__global__ void k_neg_c128(double2 *M, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        M[i] = make_double2(-M[i].x, -M[i].y);
}
// HA/HB null: B only.
int project_out(Run &r, const char *A, const char *HA, char *B, char *HB, double2 *M) {
    const size_t nn = (size_t)r.nb * r.nb;
    RK(gram(r, A, r.nb, B, r.nb, M, r.nb));
    k_neg_c128<<<blocks_for(nn), 256, 0, r.st>>>(M, nn);
    RK(rot(r, A, r.nb, M, r.nb, r.nb, B, 1));
    if (HB) RK(rot(r, HA, r.nb, M, r.nb, r.nb, HB, 1));
    return PW_OK;
}

}  // namespace

// Rinv = R^-1 with C = R^H R: the lower Cholesky factor L = R^H gives
// R^-1 = L^-H.  Uses pw_eig's Cholesky through a dedicated small routine.
namespace pwk {
cudaError_t chol_inverse_upper(double2 *C, int n, double2 *Rinv, void *work, int *d_status, cudaStream_t st);
}

namespace {
int chol_rinv(Run &r, double2 *C, int n, double2 *Rinv) {
    CKR(r.c, pwk::chol_inverse_upper(C, n, Rinv, r.eigw, r.eigstat, r.st));
    int h[2] = {0, 0};
    CKR(r.c, cudaMemcpyAsync(h, r.eigstat, sizeof(h), cudaMemcpyDeviceToHost, r.st));
    CKR(r.c, cudaStreamSynchronize(r.st));
    if (h[0]) return pwk_fail(r.c, PW_ERR_TIMEOUT, "a bounded grid barrier of the Cholesky expired");
    if (h[1]) return pwk_fail(r.c, PW_ERR_NOT_POSDEF, "cholesky(Hermitian(C)) failed: C not positive definite");
    pwk_count_launches(r.c, 4);
    return PW_OK;
}
}  // namespace
