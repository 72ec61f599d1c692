// FP64 small dense Hermitian (generalised) eigensolver on the GPU: the
// eigen(T, G) / eigvals(XHX) / eigen(S) calls of diag_LOBPCG.jl:86,185,216
// (LAPACK zhegv / zheev in the reference).
//
//   1. hermitise T and G from their upper triangles (Julia's Hermitian(A))
//   2. G = L L^H                        blocked right-looking Cholesky on
//                                       32 x 32 tiles, two grid barriers per
//                                       32-column panel (cooperative kernel)
//   3. Linv = L^-1                      blocked right-looking triangular
//                                       inverse on 32 x 32 tiles
//   4. C = Linv T Linv^H                two FP64 complex GEMMs
//   5. C = Q Tr Q^H                     Householder tridiagonalisation (LAPACK
//                                       zhetd2 conventions: H = I - tau v v^H,
//                                       real tridiagonal Tr), one grid barrier
//                                       per column (cooperative kernel)
//   6. lowest k eigenvalues of Tr       multisection on Sturm counts, one warp
//                                       per eigenvalue
//   7. eigenvectors of Tr               inverse iteration (tridiagonal LU with
//                                       partial pivoting), re-orthogonalised
//                                       (modified Gram-Schmidt) inside clusters
//                                       of near-degenerate eigenvalues, one
//                                       warp per cluster
//   8. Z = Q Ztr                        reflectors applied in reverse order,
//                                       one CTA per eigenvector
//   9. S = Linv^H Z                     FP64 complex GEMM
// The cooperative kernels synchronise with a grid barrier of their own whose
// waits are bounded; on expiry they record an error and run to completion.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "pw_eig.h"
#include "pw_launch.h"

namespace pwk {
namespace eig {

constexpr long long GSYNC_LIMIT = 1ll << 22;   // acquire polls of gsync (a few seconds)
constexpr int COOP_THREADS = 256;
constexpr int TU = 8;   // global loads kept in flight per thread in the tridiagonalisation

struct GridBar {  // barrier counter storage
    unsigned int count;
    unsigned int gen;
};

// Bounded grid-wide barrier on a monotonic counter (zeroed before the
// launch): every CTA adds one and waits until the counter reaches the
// number of CTAs times the barriers passed so far.  `tgt` is the calling
// CTA's running target (same value in every thread).
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Failure-detection test hooks, written only through pwk_test_gsync (a
// test-only export): the poll limit of every wait, and one CTA that withholds
// its arrivals so that the others' waits run out.  The library itself never
// changes them.
__device__ long long g_gsync_limit = GSYNC_LIMIT;
__device__ int g_gsync_withhold = -1;

__device__ __forceinline__ void gsync(unsigned *ctr, unsigned &tgt, int *err) {
    __syncthreads();
    tgt += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        if ((int)blockIdx.x != g_gsync_withhold) atomicAdd(ctr, 1u);
        if (!*(volatile int *)err) {
            const long long lim = g_gsync_limit;
            long long it = 0;
            while (ld_acquire_u32(ctr) < tgt) {
                if (++it > lim) {
                    atomicExch(err, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

__device__ __forceinline__ double2 cmulc_d(double2 a, double2 b) {  // conj(a) b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <typename V>
__device__ V block_sum(V v, V *red) {
    for (int o = 16; o > 0; o >>= 1) {
        if constexpr (sizeof(V) == sizeof(double2)) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        } else {
            v += __shfl_xor_sync(0xffffffffu, v, o);
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    V s = red[0];
    for (int i = 1; i < nw; ++i) {
        if constexpr (sizeof(V) == sizeof(double2)) {
            s.x += red[i].x;
            s.y += red[i].y;
        } else {
            s += red[i];
        }
    }
    return s;
}

// A (n x n, column-major): lower := conj(upper)^T, diagonal made real.
__global__ void k_herm_upper(double2 *A, int n) {
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

__global__ void k_conj_transpose(const double2 *__restrict__ A, double2 *__restrict__ B, int n) {
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        const double2 a = A[(size_t)i * n + j];
        B[t] = make_double2(a.x, -a.y);
    }
}

// ---------------------------------------------------------------- blocked
// Cholesky and triangular inverse on 32 x 32 tiles (cooperative kernels).
constexpr int TB = 32;
constexpr int TLD = TB + 1;  // shared-memory tile leading dimension (row-major)

// In-place Cholesky of the bs x bs lower block D (row-major, ld TLD).
// Returns the first failing local column + 1, or 0.  A non-positive pivot
// is replaced by a tiny one so the factorisation runs to completion.
__device__ int chol_tile(double2 *D, int bs) {
    int fail = 0;
    for (int t = 0; t < bs; ++t) {
        const double dt = D[t * TLD + t].x;
        if (!(dt > 0.0) && fail == 0) fail = t + 1;
        const double s = sqrt(fmax(dt, 1e-300)), inv = 1.0 / s;
        __syncthreads();
        for (int i = t + threadIdx.x; i < bs; i += blockDim.x)
            D[i * TLD + t] = (i == t) ? make_double2(s, 0.0) : make_double2(D[i * TLD + t].x * inv, D[i * TLD + t].y * inv);
        __syncthreads();
        for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
            const int i = idx / bs, k = idx - i * bs;
            if (k > t && i >= k) {
                const double2 p = cmulc_d(D[k * TLD + t], D[i * TLD + t]);  // D[i][t] conj(D[k][t])
                D[i * TLD + k].x -= p.x;
                D[i * TLD + k].y -= p.y;
            }
        }
        __syncthreads();
    }
    return fail;
}

// X = L^-1 for the bs x bs lower block L (both row-major, ld TLD): thread c
// solves column c by forward substitution.
__device__ void trinv_tile(const double2 *L, double2 *X, int bs) {
    for (int idx = threadIdx.x; idx < TB * TLD; idx += blockDim.x) X[idx] = make_double2(0.0, 0.0);
    __syncthreads();
    const int c = threadIdx.x;
    if (c < bs) {
        const double2 lcc = L[c * TLD + c];
        X[c * TLD + c] = make_double2(1.0 / lcc.x, 0.0);
        for (int r = c + 1; r < bs; ++r) {
            double2 s = make_double2(0.0, 0.0);
            for (int q = c; q < r; ++q) {
                const double2 p = cmul_d(L[r * TLD + q], X[q * TLD + c]);
                s.x += p.x;
                s.y += p.y;
            }
            const double il = -1.0 / L[r * TLD + r].x;
            X[r * TLD + c] = make_double2(s.x * il, s.y * il);
        }
    }
    __syncthreads();
}

// Tile (r0, c0) of the column-major n x n matrix A into T (row-major, ld
// TLD); entries outside the matrix read as zero.
__device__ void load_tile(const double2 *A, int n, int r0, int c0, double2 *T) {
#pragma unroll
    for (int idx = threadIdx.x; idx < TB * TB; idx += COOP_THREADS) {
        const int c = idx / TB, r = idx - c * TB;
        const int gr = r0 + r, gc = c0 + c;
        T[r * TLD + c] = (gr < n && gc < n) ? __ldcg(&A[(size_t)gc * n + gr]) : make_double2(0.0, 0.0);
    }
}
__device__ void store_tile(double2 *A, int n, int r0, int c0, const double2 *T) {
    for (int idx = threadIdx.x; idx < TB * TB; idx += blockDim.x) {
        const int c = idx / TB, r = idx - c * TB;
        const int gr = r0 + r, gc = c0 + c;
        if (gr < n && gc < n) A[(size_t)gc * n + gr] = T[r * TLD + c];
    }
}

// Cholesky G = L L^H, lower, in place, right-looking over 32-column panels:
//   phase 1 (every CTA): factor the diagonal block L11; the panel rows
//           below it, L21 = A21 L11^-H, by forward substitution, one warp
//           per row;
//   barrier;
//   phase 2: trailing update A22 -= L21 L21^H on lower 32 x 32 tiles
//           (cyclic over CTAs); CTA 0 stores L11;
//   barrier.
// The strict upper triangle is left as it was.  info = first failing
// column (1-based) or 0.
__global__ void __launch_bounds__(COOP_THREADS) k_chol(double2 *A, int n, unsigned *ctr, int *err, int *info) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *D = reinterpret_cast<double2 *>(sm);  // diagonal block
    double2 *Xi = D + TB * TLD;                     // 1 / diagonal of L11
    double2 *Tr = Xi + TB * TLD;                    // rows tile
    double2 *Tc = Tr + TB * TLD;                    // columns tile
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned tgt = 0;
    for (int p = 0; p < n; p += TB) {
        const int bs = min(TB, n - p);
        load_tile(A, n, p, p, D);
        __syncthreads();
        const int f = chol_tile(D, bs);
        if (f && blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(info, 0, p + f);
        if (threadIdx.x < TB) Xi[threadIdx.x] = make_double2(threadIdx.x < bs ? 1.0 / D[threadIdx.x * TLD + threadIdx.x].x : 0.0, 0.0);
        __syncthreads();
        // L21 rows by forward substitution, one warp per row i, lane t holding
        // column t:  l[t] = (a[t] - sum_{s<t} l[s] conj(L11[t][s])) / L11[t][t]
        for (int i = p + bs + blockIdx.x * nw + warp; i < n; i += gridDim.x * nw) {
            double2 acc = lane < bs ? __ldcg(&A[(size_t)(p + lane) * n + i]) : make_double2(0.0, 0.0);
            double2 l = make_double2(0.0, 0.0);
            for (int s = 0; s < bs; ++s) {
                const double is = Xi[s].x;
                const double2 ls = make_double2(__shfl_sync(0xffffffffu, acc.x, s) * is, __shfl_sync(0xffffffffu, acc.y, s) * is);
                if (lane == s) l = ls;
                if (lane > s) {
                    const double2 q = cmulc_d(D[lane * TLD + s], ls);  // ls conj(L11[lane][s])
                    acc.x -= q.x;
                    acc.y -= q.y;
                }
            }
            if (lane < bs) A[(size_t)(p + lane) * n + i] = l;
        }
        gsync(ctr, tgt, err);
        if (blockIdx.x == 0) {
            for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
                const int c = idx / bs, r = idx - c * bs;
                if (r >= c) A[(size_t)(p + c) * n + p + r] = D[r * TLD + c];
            }
        }
        const int q0 = p + bs;
        if (q0 < n) {
            const int nt = (n - q0 + TB - 1) / TB;
            const int ntiles = nt * (nt + 1) / 2;
            for (int tt = blockIdx.x; tt < ntiles; tt += gridDim.x) {
                int I = 0, rem = tt;
                while (rem > I) {
                    rem -= I + 1;
                    ++I;
                }
                const int J = rem;
                const int r0 = q0 + I * TB, c0 = q0 + J * TB;
                // Tr[r][t] = L21[r0 + r, t], Tc[c][t] = L21[c0 + c, t]
#pragma unroll
                for (int idx = threadIdx.x; idx < TB * TB; idx += COOP_THREADS) {
                    const int t = idx / TB, r = idx - t * TB;
                    Tr[r * TLD + t] = (t < bs && r0 + r < n) ? __ldcg(&A[(size_t)(p + t) * n + r0 + r]) : make_double2(0.0, 0.0);
                    Tc[r * TLD + t] = (t < bs && c0 + r < n) ? __ldcg(&A[(size_t)(p + t) * n + c0 + r]) : make_double2(0.0, 0.0);
                }
                __syncthreads();
                const int r = threadIdx.x & (TB - 1);
                for (int c = threadIdx.x / TB; c < TB; c += blockDim.x / TB) {
                    const int gr = r0 + r, gc = c0 + c;
                    if (gr < n && gc < n && gr >= gc) {
                        double2 s = make_double2(0.0, 0.0);
                        for (int t = 0; t < bs; ++t) {
                            const double2 q = cmulc_d(Tc[c * TLD + t], Tr[r * TLD + t]);
                            s.x += q.x;
                            s.y += q.y;
                        }
                        double2 *a = &A[(size_t)gc * n + gr];
                        const double2 v = __ldcg(a);
                        *a = make_double2(v.x - s.x, v.y - s.y);
                    }
                }
                __syncthreads();
            }
        }
        gsync(ctr, tgt, err);
    }
}

// X = L^-1 (L lower, column-major; X full n x n, lower result), right-looking
// over 32 x 32 tiles with X initialised to I:
//   phase 0: the diagonal block inverses DI[K] = L_KK^-1 (cyclic), X = I;
//   for each block row K:  X_KJ = DI[K] X_KJ for J <= K;  barrier;
//                          X_IJ -= L_IK X_KJ for I > K >= J;  barrier.
__global__ void __launch_bounds__(COOP_THREADS)
k_trinv(const double2 *__restrict__ L, double2 *__restrict__ X, double2 *__restrict__ DI, int n, unsigned *ctr, int *err) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *Ta = reinterpret_cast<double2 *>(sm);
    double2 *Tb = Ta + TB * TLD;
    double2 *Tx = Tb + TB * TLD;
    unsigned tgt = 0;
    const int nbk = (n + TB - 1) / TB;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)n * n; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / n), i = (int)(t - (size_t)j * n);
        X[t] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
    for (int K = blockIdx.x; K < nbk; K += gridDim.x) {
        load_tile(L, n, K * TB, K * TB, Ta);
        __syncthreads();
        trinv_tile(Ta, Tb, min(TB, n - K * TB));
        for (int idx = threadIdx.x; idx < TB * TB; idx += blockDim.x) DI[(size_t)K * TB * TB + idx] = Tb[(idx / TB) * TLD + idx % TB];
        __syncthreads();
    }
    gsync(ctr, tgt, err);
    const int r = threadIdx.x & (TB - 1);
    for (int K = 0; K < nbk; ++K) {
        // X_KJ = DI[K] X_KJ
        for (int J = blockIdx.x; J <= K; J += gridDim.x) {
            for (int idx = threadIdx.x; idx < TB * TB; idx += blockDim.x) Ta[(idx / TB) * TLD + idx % TB] = DI[(size_t)K * TB * TB + idx];
            load_tile(X, n, K * TB, J * TB, Tx);
            __syncthreads();
            for (int c = threadIdx.x / TB; c < TB; c += blockDim.x / TB) {
                double2 s = make_double2(0.0, 0.0);
                for (int q = 0; q <= r; ++q) {
                    const double2 p = cmul_d(Ta[r * TLD + q], Tx[q * TLD + c]);
                    s.x += p.x;
                    s.y += p.y;
                }
                Tb[r * TLD + c] = s;
            }
            __syncthreads();
            store_tile(X, n, K * TB, J * TB, Tb);
            __syncthreads();
        }
        gsync(ctr, tgt, err);
        // X_IJ -= L_IK X_KJ
        const int ni = nbk - K - 1, nj = K + 1;
        for (int tt = blockIdx.x; tt < ni * nj; tt += gridDim.x) {
            const int I = K + 1 + tt / nj, J = tt % nj;
            load_tile(L, n, I * TB, K * TB, Ta);
            load_tile(X, n, K * TB, J * TB, Tx);
            load_tile(X, n, I * TB, J * TB, Tb);
            __syncthreads();
            for (int c = threadIdx.x / TB; c < TB; c += blockDim.x / TB) {
                double2 s = Tb[r * TLD + c];
                for (int q = 0; q < TB; ++q) {
                    const double2 p = cmul_d(Ta[r * TLD + q], Tx[q * TLD + c]);
                    s.x -= p.x;
                    s.y -= p.y;
                }
                Tb[r * TLD + c] = s;
            }
            __syncthreads();
            store_tile(X, n, I * TB, J * TB, Tb);
            __syncthreads();
        }
        gsync(ctr, tgt, err);
    }
}

// Householder tridiagonalisation of the Hermitian C (full storage), LAPACK
// zhetd2 (lower) conventions: H_j = I - tau_j v_j v_j^H with v_j[j+1] = 1,
// real tridiagonal (d, e); v_j is left in C[j+2:n, j].  One grid barrier per
// column:
//   phase M (distributed): the owner of each trailing column i > j applies
//     the previous step's rank-2 update  A -= v w^H + w v^H  to rows > j and,
//     in the same pass, forms y_i = (column i)^H v_j;
//   barrier;
//   phase R (every CTA, redundantly): w_j = tau y + alpha v_j with
//     alpha = -tau/2 (tau y)^H v_j; the next column j+1 is read, given the
//     step-j update, and its Householder vector v_{j+1} formed.
// Every CTA therefore holds v_j, w_j, v_{j-1}, w_{j-1} in shared memory and
// the trailing matrix is read and written once per column.  y alternates
// between two buffers so that a CTA running ahead into the next phase M
// cannot overwrite values a slower CTA still reads.
__global__ void __launch_bounds__(COOP_THREADS)
k_tridiag(double2 *C, int n, double *d, double *e, double2 *tau, double2 *ybuf, unsigned *ctr, int *err) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *vc = reinterpret_cast<double2 *>(sm);  // v_j         [n]
    double2 *vp = vc + n;                           // v_{j-1}     [n]
    double2 *wp = vp + n;                           // w_{j-1}     [n]
    double2 *red = wp + n;                          // [32]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned tgt = 0;
    double2 tj = make_double2(0.0, 0.0);

    // Householder vector of x = vc[j+1 .. n) in place (vc[j] := 0,
    // vc[j+1] := 1); returns tau.  CTA 0 records e[j] = beta and tau[j].
    auto householder = [&](int j) -> double2 {
        double s2 = 0.0;
        for (int i = j + 2 + threadIdx.x; i < n; i += blockDim.x) s2 += vc[i].x * vc[i].x + vc[i].y * vc[i].y;
        s2 = block_sum<double>(s2, (double *)red);
        const double2 alpha = vc[j + 1];
        double2 t, scal;
        double beta;
        if (s2 == 0.0 && alpha.y == 0.0) {
            t = make_double2(0.0, 0.0);
            beta = alpha.x;
            scal = make_double2(0.0, 0.0);
        } else {
            beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2), alpha.x);
            t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
            const double ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
            scal = make_double2(ar / den, -ai / den);
        }
        __syncthreads();  // everyone has read vc[j+1]
        for (int i = j + threadIdx.x; i < n; i += blockDim.x)
            vc[i] = (i == j) ? make_double2(0.0, 0.0) : (i == j + 1) ? make_double2(1.0, 0.0) : cmul_d(vc[i], scal);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            e[j] = beta;
            tau[j] = t;
        }
        __syncthreads();
        return t;
    };

    // column 0
    for (int i = threadIdx.x; i < n; i += blockDim.x) vc[i] = __ldcg(&C[i]);
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) d[0] = vc[0].x;
    if (n >= 2) tj = householder(0);

    for (int j = 0; j < n - 1; ++j) {
        double2 *yb = ybuf + (size_t)(j & 1) * n;
        // ---- phase M: update owned columns i > j with (v_{j-1}, w_{j-1}), y_i = col_i^H v_j
        for (int i = j + 1 + blockIdx.x + gridDim.x * warp; i < n; i += gridDim.x * nw) {
            double2 *col = C + (size_t)i * n;
            double2 acc = make_double2(0.0, 0.0);
            // (v, w) = (0, 0) at j = 0: no previous update
            const double2 cw = j > 0 ? make_double2(wp[i].x, -wp[i].y) : make_double2(0.0, 0.0);
            const double2 cv = j > 0 ? make_double2(vp[i].x, -vp[i].y) : make_double2(0.0, 0.0);
            // TU loads in flight per lane: the column streams from L2
            for (int r0 = j + 1 + lane; r0 < n; r0 += 32 * TU) {
                double2 a[TU];
#pragma unroll
                for (int u = 0; u < TU; ++u) {
                    const int r = r0 + 32 * u;
                    a[u] = r < n ? __ldcg(&col[r]) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < TU; ++u) {
                    const int r = r0 + 32 * u;
                    if (r < n) {
                        if (j > 0) {
                            const double2 p = cmul_d(vp[r], cw), q = cmul_d(wp[r], cv);
                            a[u].x -= p.x + q.x;
                            a[u].y -= p.y + q.y;
                            col[r] = a[u];
                        }
                        const double2 s = cmulc_d(a[u], vc[r]);
                        acc.x += s.x;
                        acc.y += s.y;
                    }
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
            }
            if (lane == 0) yb[i] = acc;
        }
        gsync(ctr, tgt, err);
        // ---- phase R (redundant).  Column j is no longer read by anyone:
        // its owner stores v_j there for the back-transformation.
        if ((j % gridDim.x) == blockIdx.x)
            for (int i = j + 2 + threadIdx.x; i < n; i += blockDim.x) C[(size_t)j * n + i] = vc[i];
        // v_{j-1}, w_{j-1} are dead now.  One batch of loads brings in both
        // y (scaled by tau, into wp) and the raw next column j+1 (into vp).
        const int c1 = j + 1;
        const double2 *col = C + (size_t)c1 * n;
        for (int base = threadIdx.x; base < n; base += blockDim.x * TU) {
            double2 ya[TU], ca[TU];
#pragma unroll
            for (int u = 0; u < TU; ++u) {
                const int i = base + u * blockDim.x;
                ya[u] = (i > j && i < n) ? __ldcg(&yb[i]) : make_double2(0.0, 0.0);
                ca[u] = (i >= c1 && i < n) ? __ldcg(&col[i]) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < TU; ++u) {
                const int i = base + u * blockDim.x;
                if (i < n) {
                    wp[i] = cmul_d(tj, ya[u]);
                    vp[i] = ca[u];
                }
            }
        }
        __syncthreads();
        // w_j = tau y + alpha v_j, alpha = -tau/2 (tau y)^H v_j
        double2 yv = make_double2(0.0, 0.0);
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double2 s = cmulc_d(wp[i], vc[i]);
            yv.x += s.x;
            yv.y += s.y;
        }
        yv = block_sum<double2>(yv, red);
        const double2 al = cmul_d(make_double2(-0.5 * tj.x, -0.5 * tj.y), yv);
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double2 p = cmul_d(al, vc[i]);
            wp[i].x += p.x;
            wp[i].y += p.y;
        }
        __syncthreads();
        // v_j becomes v_{j-1} for the next step; the next column (in the
        // old v_{j-1} buffer) becomes vc and gets the step-j update
        double2 *t = vp;
        vp = vc;
        vc = t;
        const double2 cw = make_double2(wp[c1].x, -wp[c1].y), cv = make_double2(vp[c1].x, -vp[c1].y);
        for (int r = c1 + threadIdx.x; r < n; r += blockDim.x) {
            const double2 p = cmul_d(vp[r], cw), q = cmul_d(wp[r], cv);
            vc[r].x -= p.x + q.x;
            vc[r].y -= p.y + q.y;
        }
        __syncthreads();
        if (blockIdx.x == 0 && threadIdx.x == 0) d[c1] = vc[c1].x;
        if (c1 < n - 1) tj = householder(c1);
    }
}

__device__ int sturm_count(const double *d, const double *e, int n, double x, double pivmin) {
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    int c = q < 0.0;
    for (int i = 1; i < n; ++i) {
        q = (d[i] - x) - e[i - 1] * e[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        c += q < 0.0;
    }
    return c;
}

// lowest k eigenvalues of the real symmetric tridiagonal (d, e), ascending.
// Multisection: one warp per eigenvalue; each round the 32 lanes take Sturm
// counts at 32 interior points of the current interval [a, b], which then
// shrinks 33-fold to the sub-interval that holds eigenvalue i.
__global__ void k_bisect(const double *__restrict__ d, const double *__restrict__ e, int n, int k, double *__restrict__ lam,
                         double *__restrict__ nrm_out) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= k) return;
    double lo = 1e300, hi = -1e300, emax2 = 0.0;
    for (int r = lane; r < n; r += 32) {
        const double rad = (r > 0 ? fabs(e[r - 1]) : 0.0) + (r < n - 1 ? fabs(e[r]) : 0.0);
        lo = fmin(lo, d[r] - rad);
        hi = fmax(hi, d[r] + rad);
        if (r < n - 1) emax2 = fmax(emax2, e[r] * e[r]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        emax2 = fmax(emax2, __shfl_xor_sync(0xffffffffu, emax2, o));
    }
    const double nrm = fmax(fabs(lo), fabs(hi));
    const double pivmin = fmax(2.2250738585072014e-308, 2.2250738585072014e-308 * emax2) * 4.0;
    double a = lo - 1e-14 * nrm - 1e-300, b = hi + 1e-14 * nrm + 1e-300;
    for (int it = 0; it < 64; ++it) {
        if (b - a <= 2.0 * 2.220446049250313e-16 * fmax(fabs(a), fabs(b))) break;
        const double h = (b - a) / 33.0;
        const double x = fmin(fmax(a + (lane + 1) * h, a), b);
        const bool above = sturm_count(d, e, n, x, pivmin) > i;   // eigenvalue i lies below x
        const unsigned m = __ballot_sync(0xffffffffu, above);
        const int f = m ? __ffs(m) - 1 : 32;                       // first sample point above it (warp-uniform)
        const double xl = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
        const double xr = __shfl_sync(0xffffffffu, x, f < 32 ? f : 31);
        const double na = f > 0 ? xl : a, nb = f < 32 ? xr : b;
        if (na == a && nb == b) break;  // no representable progress
        a = na;
        b = nb;
    }
    if (lane == 0) {
        lam[i] = 0.5 * (a + b);
        if (i == 0) *nrm_out = nrm;
    }
}

// LU factorisation with partial pivoting of (Tr - lam I) (LAPACK dgttrf
// pattern): rows i and i+1 swap when |sub| > |pivot|.  Outputs, per row:
// rd = 1 / U[i][i], du = U[i][i+1], du2 = U[i][i+2], lm = multiplier,
// pv = 1 where rows i, i+1 were swapped.  A zero pivot is replaced by a
// tiny one (the shift sits on an eigenvalue to working precision).
__device__ void tri_factor(const double *d, const double *e, int n, double lam, double *rd, double *du, double *du2,
                           double *lm, unsigned char *pv) {
    double di = d[0] - lam, ui = n > 1 ? e[0] : 0.0;
    for (int i = 0; i < n - 1; ++i) {
        const double sub = e[i];
        const double dn = d[i + 1] - lam, un = (i + 1 < n - 1) ? e[i + 1] : 0.0;
        if (fabs(di) >= fabs(sub)) {
            if (di == 0.0) di = 1e-300;
            const double f = sub / di;
            rd[i] = 1.0 / di;
            du[i] = ui;
            du2[i] = 0.0;
            lm[i] = f;
            pv[i] = 0;
            di = dn - f * ui;
            ui = un;
        } else {
            const double f = di / sub;
            rd[i] = 1.0 / sub;
            du[i] = dn;
            du2[i] = un;
            lm[i] = f;
            pv[i] = 1;
            di = ui - f * dn;
            ui = -f * un;
        }
    }
    if (di == 0.0) di = 1e-300;
    rd[n - 1] = 1.0 / di;
    du[n - 1] = 0.0;
    du2[n - 1] = 0.0;
}

// b := (Tr - lam I)^-1 b with the factorisation of tri_factor.
__device__ void tri_solve(int n, const double *rd, const double *du, const double *du2, const double *lm,
                          const unsigned char *pv, double *b) {
    double bi = b[0];
    for (int i = 0; i < n - 1; ++i) {
        const double bn = b[i + 1];
        if (pv[i]) {
            b[i] = bn;
            bi = bi - lm[i] * bn;
        } else {
            b[i] = bi;
            bi = bn - lm[i] * bi;
        }
    }
    b[n - 1] = bi;
    double x2 = 0.0, x1 = b[n - 1] * rd[n - 1];
    b[n - 1] = x1;
    for (int i = n - 2; i >= 0; --i) {
        const double x = (b[i] - du[i] * x1 - du2[i] * x2) * rd[i];
        b[i] = x;
        x2 = x1;
        x1 = x;
    }
}

// One warp per cluster of near-degenerate eigenvalues (gap <= ortol):
// inverse iteration for each member (one factorisation, INVIT_STEPS solves),
// re-orthogonalised against the earlier members of its cluster.  The
// factorisation and the iterate live in shared memory (lane 0 runs the
// sequential recurrences).  Z: n x k real (column-major).
constexpr int INVIT_STEPS = 3;
__global__ void k_invit(const double *__restrict__ d, const double *__restrict__ e, int n, int k,
                        const double *__restrict__ lam, const double *__restrict__ nrmp, double reltol,
                        double *__restrict__ Z) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const int wid = blockIdx.x * (blockDim.x >> 5) + wl;
    double *rd = reinterpret_cast<double *>(sm) + (size_t)wl * 5 * n;
    double *du = rd + n, *du2 = du + n, *lm = du2 + n, *x = lm + n;
    unsigned char *pv = sm + (size_t)(blockDim.x >> 5) * 5 * n * sizeof(double) + (size_t)wl * n;
    if (wid >= k) return;
    const double nrm = *nrmp;
    const double ortol = reltol * nrm;
    const double eps = 2.220446049250313e-16;
    // a warp owns eigenvalue wid only if it starts a cluster
    if (wid > 0 && lam[wid] - lam[wid - 1] <= ortol) return;
    int end = wid + 1;
    while (end < k && lam[end] - lam[end - 1] <= ortol) ++end;
    double lprev = 0.0;
    for (int i = wid; i < end; ++i) {
        double li = lam[i];
        if (i > wid && li - lprev < 10.0 * eps * nrm) li = lprev + 10.0 * eps * nrm;  // separate degenerate shifts
        lprev = li;
        // deterministic pseudo-random start
        for (int r = lane; r < n; r += 32) {
            unsigned int h = (unsigned int)(r * 2654435761u) ^ (unsigned int)(i * 2246822519u + 12345u);
            h ^= h >> 15;
            h *= 2246822519u;
            h ^= h >> 13;
            x[r] = ((double)(h & 0xFFFFFF) / 16777216.0) - 0.5;
        }
        if (lane == 0) tri_factor(d, e, n, li, rd, du, du2, lm, pv);
        __syncwarp();
        for (int it = 0; it < INVIT_STEPS; ++it) {
            if (lane == 0) tri_solve(n, rd, du, du2, lm, pv, x);
            __syncwarp();
            for (int jj = wid; jj < i; ++jj) {  // modified Gram-Schmidt inside the cluster
                const double *q = Z + (size_t)jj * n;
                double s = 0.0;
                for (int r = lane; r < n; r += 32) s += q[r] * x[r];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                for (int r = lane; r < n; r += 32) x[r] -= s * q[r];
                __syncwarp();
            }
            double s = 0.0;
            for (int r = lane; r < n; r += 32) s += x[r] * x[r];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            const double inv = 1.0 / sqrt(fmax(s, 1e-300));
            for (int r = lane; r < n; r += 32) x[r] *= inv;
            __syncwarp();
        }
        double *z = Z + (size_t)i * n;
        for (int r = lane; r < n; r += 32) z[r] = x[r];
        __syncwarp();
    }
}

// shared memory of k_invit per warp
inline size_t invit_smem_per_warp(int n) { return (size_t)n * (5 * sizeof(double) + 1); }

// Z[:, c] = Q Ztr[:, c], Q = H_0 H_1 ... H_{n-2}: reflectors in reverse order.
__global__ void k_backtr(const double2 *__restrict__ C, const double2 *__restrict__ tau, int n,
                         const double *__restrict__ Zt, double2 *__restrict__ Z) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *z = reinterpret_cast<double2 *>(sm);
    double2 *red = z + n;
    const int c = blockIdx.x;
    for (int i = threadIdx.x; i < n; i += blockDim.x) z[i] = make_double2(Zt[(size_t)c * n + i], 0.0);
    __syncthreads();
    for (int j = n - 2; j >= 0; --j) {
        const double2 t = tau[j];
        if (t.x == 0.0 && t.y == 0.0) continue;
        const double2 *vj = C + (size_t)j * n;  // v_j[i] at row i >= j+1, v_j[j+1] = 1
        double2 acc = make_double2(0.0, 0.0);
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double2 vi = (i == j + 1) ? make_double2(1.0, 0.0) : vj[i];
            const double2 p = cmulc_d(vi, z[i]);
            acc.x += p.x;
            acc.y += p.y;
        }
        acc = block_sum<double2>(acc, red);
        const double2 f = cmul_d(t, acc);
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double2 vi = (i == j + 1) ? make_double2(1.0, 0.0) : vj[i];
            const double2 p = cmul_d(vi, f);
            z[i].x -= p.x;
            z[i].y -= p.y;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) Z[(size_t)c * n + i] = z[i];
}

int blocks_for(size_t total) {
    size_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return b < 1 ? 1 : (int)b;
}

cudaError_t coop_blocks(const void *fn, size_t smem, int *nblk) {
    int dev = 0, sms = 0, per = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, COOP_THREADS, smem)) != cudaSuccess) return e;
    if (per < 1) return cudaErrorCooperativeLaunchTooLarge;
    *nblk = sms * std::min(per, 1);  // one CTA per SM keeps the barrier cheap
    return cudaSuccess;
}

}  // namespace eig

using namespace eig;

size_t eig_work_bytes(int n, int k) {
    const size_t nn = (size_t)n * n * sizeof(double2);
    return 2 * nn                                     // L^-1, scratch n x n
           + (size_t)2 * n * sizeof(double2)          // y (two buffers)
           + (size_t)(3 * n) * sizeof(double)         // d, e, lam
           + (size_t)n * sizeof(double2)              // tau
           + (size_t)n * k * sizeof(double)           // Ztr
           + (size_t)n * k * sizeof(double2)          // Z
           + (size_t)((n + TB - 1) / TB) * TB * TB * sizeof(double2)   // inverse diagonal tiles
           + 16 * 256;                                // barrier, status, norm + 256-byte rounding of 13 pieces
}

// L = chol(G) in place (lower), Linv = L^-1.  ctr: barrier counter, err:
// [0] barrier expiry, [1] first failing Cholesky column (1-based).
cudaError_t chol_and_inverse(double2 *G, int n, double2 *Linv, double2 *DI, unsigned *ctr, int *err, cudaStream_t st) {
    cudaError_t e_;
    const int nt = (n + TB - 1) / TB;
    {
        const size_t smem = 4 * (size_t)TB * TLD * sizeof(double2);
        int nblk = 0;
        if ((e_ = coop_blocks((const void *)k_chol, smem, &nblk)) != cudaSuccess) return e_;
        nblk = std::max(1, std::min(nblk, nt * (nt + 1) / 2));
        if ((e_ = cudaMemsetAsync(ctr, 0, sizeof(unsigned), st)) != cudaSuccess) return e_;
        int *info = err + 1;
        void *args[] = {(void *)&G, (void *)&n, (void *)&ctr, (void *)&err, (void *)&info};
        if ((e_ = cudaLaunchCooperativeKernel((const void *)k_chol, nblk, COOP_THREADS, args, smem, st)) != cudaSuccess) return e_;
    }
    {
        const size_t smem = 3 * (size_t)TB * TLD * sizeof(double2);
        int nblk = 0;
        if ((e_ = coop_blocks((const void *)k_trinv, smem, &nblk)) != cudaSuccess) return e_;
        nblk = std::max(1, std::min(nblk, std::max(nt, (nt * nt + 3) / 4)));
        if ((e_ = cudaMemsetAsync(ctr, 0, sizeof(unsigned), st)) != cudaSuccess) return e_;
        void *args[] = {(void *)&G, (void *)&Linv, (void *)&DI, (void *)&n, (void *)&ctr, (void *)&err};
        if ((e_ = cudaLaunchCooperativeKernel((const void *)k_trinv, nblk, COOP_THREADS, args, smem, st)) != cudaSuccess) return e_;
    }
    return cudaSuccess;
}

// flag[0] = 1 if any diagonal or off-diagonal entry of the tridiagonal
// matrix is not finite
__global__ void k_check_finite(const double *__restrict__ d, const double *__restrict__ e, int n, int *flag) {
    bool bad = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) bad |= !isfinite(d[i]) || (i + 1 < n && !isfinite(e[i]));
    if (__syncthreads_or(bad) && threadIdx.x == 0) *flag = 1;
}

cudaError_t hegv_lowest(double2 *T, double2 *G, int n, int k, double *lam_out, double2 *S, void *work, size_t work_bytes,
                        void *gemm_ws, int *d_status, cudaStream_t st) {
    if (n <= 0 || k <= 0 || k > n || work_bytes < eig_work_bytes(n, k)) return cudaErrorInvalidValue;
    unsigned char *p = (unsigned char *)work;
    auto take = [&](size_t bytes) {
        unsigned char *q = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)q;
    };
    const size_t nn = (size_t)n * n;
    double2 *Linv = (double2 *)take(nn * sizeof(double2));
    double2 *M1 = (double2 *)take(nn * sizeof(double2));
    double2 *xg = (double2 *)take(2 * (size_t)n * sizeof(double2));
    double *d = (double *)take(n * sizeof(double));
    double *e = (double *)take(n * sizeof(double));
    double *lam = (double *)take(n * sizeof(double));
    double2 *tau = (double2 *)take(n * sizeof(double2));
    double *Zt = (double *)take((size_t)n * k * sizeof(double));
    double2 *Z = (double2 *)take((size_t)n * k * sizeof(double2));
    double2 *DI = (double2 *)take((size_t)((n + TB - 1) / TB) * TB * TB * sizeof(double2));
    GridBar *gb = (GridBar *)take(sizeof(GridBar));
    int *err = (int *)take(sizeof(int) * 4);
    double *nrm = (double *)take(sizeof(double));
    unsigned *ctr = &gb->count;
    cudaError_t e_;
    if ((e_ = cudaMemsetAsync(gb, 0, sizeof(GridBar), st)) != cudaSuccess) return e_;
    if ((e_ = cudaMemsetAsync(err, 0, sizeof(int) * 4, st)) != cudaSuccess) return e_;
    const int nb = blocks_for(nn);
    k_herm_upper<<<nb, 256, 0, st>>>(T, n);
    double2 *Cm = T;
    if (G) {
        k_herm_upper<<<nb, 256, 0, st>>>(G, n);
        if ((e_ = chol_and_inverse(G, n, Linv, DI, ctr, err, st)) != cudaSuccess) return e_;
        // C = Linv T Linv^H: Linv lower triangular, only C's upper triangle
        // is read (n = 1440: the two full products took 3.06 ms)
        if ((e_ = gemm_nn<double>(n, n, n, Linv, n, T, n, M1, n, 0, st, 1)) != cudaSuccess) return e_;
        k_conj_transpose<<<nb, 256, 0, st>>>(Linv, G, n);  // G no longer needed: holds Linv^H
        if ((e_ = gemm_nn<double>(n, n, n, M1, n, G, n, T, n, 0, st, 2)) != cudaSuccess) return e_;
        k_herm_upper<<<nb, 256, 0, st>>>(T, n);
    }
    {
        const size_t smem = (size_t)(3 * n + 32) * sizeof(double2);
        int nblk = 0;
        if ((e_ = coop_blocks((const void *)k_tridiag, smem, &nblk)) != cudaSuccess) return e_;
        // about one trailing column per warp at the start: fewer CTAs keep
        // the per-column barrier cheap for small n
        nblk = std::max(1, std::min(nblk, (n + 7) / 8));
        if ((e_ = cudaMemsetAsync(ctr, 0, sizeof(unsigned), st)) != cudaSuccess) return e_;
        void *args[] = {(void *)&Cm, (void *)&n, (void *)&d, (void *)&e, (void *)&tau, (void *)&xg, (void *)&ctr, (void *)&err};
        if ((e_ = cudaLaunchCooperativeKernel((const void *)k_tridiag, nblk, COOP_THREADS, args, smem, st)) != cudaSuccess)
            return e_;
    }
    // a non-finite T or G reaches the tridiagonal matrix: report it (the
    // Sturm counts would otherwise turn it into finite, meaningless values)
    k_check_finite<<<1, 256, 0, st>>>(d, e, n, err + 2);
    k_bisect<<<(k + 7) / 8, 256, 0, st>>>(d, e, n, k, lam, nrm);
    if ((e_ = cudaMemcpyAsync(lam_out, lam, k * sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e_;
    if (S) {
        {
            // as many warps per CTA as fit in about 200 KB of shared memory
            const size_t per = invit_smem_per_warp(n);
            const int wpc = (int)std::max<size_t>(1, std::min<size_t>(8, (200u << 10) / per));
            const size_t smem = ((per * wpc) + 15) & ~(size_t)15;
            if (smem > 48 * 1024 &&
                (e_ = cudaFuncSetAttribute((const void *)k_invit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                    cudaSuccess)
                return e_;
            k_invit<<<(k + wpc - 1) / wpc, 32 * wpc, smem, st>>>(d, e, n, k, lam, nrm, 1e-7, Zt);
        }
        const size_t smem = (size_t)(n + 32) * sizeof(double2);
        if (smem > 48 * 1024 &&
            (e_ = cudaFuncSetAttribute((const void *)k_backtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
            return e_;
        k_backtr<<<k, 256, smem, st>>>(Cm, tau, n, Zt, G ? Z : S);
        if (G) {
            // S = Linv^H Z  (Linv^H sits in G)
            if ((e_ = gemm_nn<double>(n, k, n, G, n, Z, n, S, n, 0, st, 3)) != cudaSuccess) return e_;
        }
    }
    if ((e_ = cudaGetLastError()) != cudaSuccess) return e_;
    // status: [0] barrier expiry, [1] Cholesky breakdown column (1-based),
    // [2] non-finite tridiagonal matrix
    return cudaMemcpyAsync(d_status, err, 3 * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

cudaError_t chol_inverse_upper(double2 *C, int n, double2 *Rinv, void *work, int *d_status, cudaStream_t st) {
    unsigned char *p = (unsigned char *)work;
    double2 *Linv = (double2 *)p;
    p += (((size_t)n * n * sizeof(double2)) + 255) & ~(size_t)255;
    double2 *DI = (double2 *)p;
    p += (((size_t)((n + TB - 1) / TB) * TB * TB * sizeof(double2)) + 255) & ~(size_t)255;
    unsigned *ctr = (unsigned *)p;
    p += 256;
    int *err = (int *)p;
    cudaError_t e_;
    if ((e_ = cudaMemsetAsync(err, 0, sizeof(int) * 4, st)) != cudaSuccess) return e_;
    const int nb = blocks_for((size_t)n * n);
    k_herm_upper<<<nb, 256, 0, st>>>(C, n);
    if ((e_ = chol_and_inverse(C, n, Linv, DI, ctr, err, st)) != cudaSuccess) return e_;
    k_conj_transpose<<<nb, 256, 0, st>>>(Linv, Rinv, n);
    if ((e_ = cudaGetLastError()) != cudaSuccess) return e_;
    return cudaMemcpyAsync(d_status, err, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

}  // namespace pwk

// Test-only export (not in pwb200.h): sets the grid-barrier poll limit
// (limit <= 0 restores the default) and the CTA that withholds its arrivals
// (-1: none) on `device`, for the tests that make a bounded wait expire
// without faulting or hanging the GPU.
extern "C" int pwk_test_gsync(int device, long long limit, int withhold_cta) {
    if (cudaSetDevice(device) != cudaSuccess) return 2;
    const long long lim = limit > 0 ? limit : pwk::eig::GSYNC_LIMIT;
    if (cudaMemcpyToSymbol(pwk::eig::g_gsync_limit, &lim, sizeof(lim)) != cudaSuccess) return 2;
    if (cudaMemcpyToSymbol(pwk::eig::g_gsync_withhold, &withhold_cta, sizeof(withhold_cta)) != cudaSuccess) return 2;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}
