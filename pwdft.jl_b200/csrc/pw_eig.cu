// FP64 small dense Hermitian (generalised) eigensolver on the GPU: the
// eigen(T, G) / eigvals(XHX) / eigen(S) calls of diag_LOBPCG.jl:86,185,216
// (LAPACK zhegv / zheev in the reference).
//
//   1. hermitise T and G from their upper triangles (Julia's Hermitian(A))
//   2. G = L L^H                        Cholesky, right-looking, one column per
//                                       grid-wide step (cooperative kernel)
//   3. Linv = L^-1                      one warp per column, column-oriented
//                                       forward substitution
//   4. C = Linv T Linv^H                two FP64 complex GEMMs
//   5. C = Q Tr Q^H                     Householder tridiagonalisation (LAPACK
//                                       zhetd2 conventions: H = I - tau v v^H,
//                                       real tridiagonal Tr), two grid-wide
//                                       steps per column (cooperative kernel)
//   6. lowest k eigenvalues of Tr       bisection on Sturm counts, one thread
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

constexpr long long BARRIER_LIMIT = 1ll << 24;
constexpr int COOP_THREADS = 256;

struct GridBar {
    unsigned int count;
    unsigned int gen;
};

// Bounded grid-wide barrier (all CTAs are co-resident: cooperative launch).
__device__ __forceinline__ void grid_barrier(GridBar *gb, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = &gb->gen;
        const unsigned int g = *vgen;
        __threadfence();
        if (atomicAdd(&gb->count, 1u) == gridDim.x - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else if (!*(volatile int *)err) {
            long long it = 0;
            while (*vgen == g) {
                if (++it > BARRIER_LIMIT) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
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

// Cholesky, lower, in place.  Step j: every CTA reads the final column j,
// updates the columns k > j it owns (k mod gridDim == blockIdx) with
// A[i][k] -= A[i][j] conj(A[k][j]) / A[j][j]; the owner of column j-1 scales
// it by 1/sqrt(A[j-1][j-1]) (no CTA reads column j-1 any more).
__global__ void __launch_bounds__(COOP_THREADS) k_chol(double2 *A, int n, GridBar *gb, int *err, int *info) {
    for (int j = 0; j < n; ++j) {
        const double djj = __ldcg(&A[(size_t)j * n + j]).x;
        if (!(djj > 0.0)) {
            if (threadIdx.x == 0 && blockIdx.x == 0) atomicCAS(info, 0, j + 1);
        }
        const double inv = djj > 0.0 ? 1.0 / djj : 0.0;
        const double2 *colj = A + (size_t)j * n;
        for (int k = j + 1 + blockIdx.x; k < n; k += gridDim.x) {
            const double2 akj = __ldcg(&colj[k]);
            double2 *colk = A + (size_t)k * n;
            for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
                const double2 aij = __ldcg(&colj[i]);
                // aij * conj(akj) / djj
                const double2 p = make_double2((aij.x * akj.x + aij.y * akj.y) * inv, (aij.y * akj.x - aij.x * akj.y) * inv);
                colk[i].x -= p.x;
                colk[i].y -= p.y;
            }
        }
        if (j > 0 && ((j - 1) % gridDim.x) == blockIdx.x) {
            double2 *c = A + (size_t)(j - 1) * n;
            const double s = 1.0 / sqrt(fmax(c[j - 1].x, 1e-300));
            for (int i = j - 1 + threadIdx.x; i < n; i += blockDim.x) c[i] = make_double2(c[i].x * s, c[i].y * s);
        }
        grid_barrier(gb, err);
    }
    if (((n - 1) % gridDim.x) == blockIdx.x) {
        double2 *c = A + (size_t)(n - 1) * n;
        const double s = 1.0 / sqrt(fmax(c[n - 1].x, 1e-300));
        if (threadIdx.x == 0) c[n - 1] = make_double2(c[n - 1].x * s, 0.0);
    }
}

// Linv = L^-1 (lower): warp w solves L x = e_c for column c, column-oriented.
__global__ void k_trinv_lower(const double2 *__restrict__ L, double2 *__restrict__ X, int n) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= n) return;
    double2 *x = X + (size_t)c * n;
    for (int i = lane; i < n; i += 32) x[i] = make_double2(i == c ? 1.0 : 0.0, 0.0);
    __syncwarp();
    for (int j = c; j < n; ++j) {
        const double2 ljj = L[(size_t)j * n + j];
        double2 xj = x[j];
        const double inv = 1.0 / ljj.x;  // real positive diagonal
        xj = make_double2(xj.x * inv, xj.y * inv);
        __syncwarp();
        if (lane == 0) x[j] = xj;
        const double2 *lj = L + (size_t)j * n;
        for (int i = j + 1 + lane; i < n; i += 32) {
            const double2 p = cmul_d(lj[i], xj);
            x[i].x -= p.x;
            x[i].y -= p.y;
        }
        __syncwarp();
    }
}

// Householder tridiagonalisation of the Hermitian C (full storage), LAPACK
// zhetd2 (lower) conventions.  Outputs d (n), e (n-1), tau (n-1); the vector
// v_j (v_j[0] = 1 implicit) is stored in C[j+2:n, j], written one step late.
__global__ void __launch_bounds__(COOP_THREADS)
k_tridiag(double2 *C, int n, double *d, double *e, double2 *tau, double2 *xg, GridBar *gb, int *err) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *v = reinterpret_cast<double2 *>(sm);  // [n]
    double2 *w = v + n;                            // [n]
    double2 *red = w + n;                          // [32]
    double2 *vprev = red + 32;                     // [n]   v of the previous step (owner writes it back)
    int prev_m = 0;
    for (int j = 0; j < n - 1; ++j) {
        const int m = n - j - 1;
        const double2 *cj = C + (size_t)j * n + (j + 1);  // x = C[j+1:n, j]
        // --- Householder vector (every CTA, redundantly)
        double s2 = 0.0;
        for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) {
            const double2 c = __ldcg(&cj[i]);
            s2 += c.x * c.x + c.y * c.y;
        }
        s2 = block_sum<double>(s2, (double *)red);
        const double2 alpha = __ldcg(&cj[0]);
        double2 t;
        double beta;
        double2 scal;
        if (s2 == 0.0 && alpha.y == 0.0) {
            t = make_double2(0.0, 0.0);
            beta = alpha.x;
            scal = make_double2(0.0, 0.0);
        } else {
            beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + s2), alpha.x);
            t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
            // 1 / (alpha - beta)
            const double ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
            scal = make_double2(ar / den, -ai / den);
        }
        for (int i = threadIdx.x; i < m; i += blockDim.x) v[i] = (i == 0) ? make_double2(1.0, 0.0) : cmul_d(__ldcg(&cj[i]), scal);
        // the owner of column j-1 stores v_{j-1}; record d, e, tau
        if (j > 0 && ((j - 1) % gridDim.x) == blockIdx.x) {
            double2 *cp = C + (size_t)(j - 1) * n + j;
            for (int i = 1 + threadIdx.x; i < prev_m; i += blockDim.x) cp[i] = vprev[i];
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            d[j] = __ldcg(&C[(size_t)j * n + j]).x;
            e[j] = beta;
            tau[j] = t;
        }
        __syncthreads();
        // --- x = tau * A22 v, rows owned cyclically; row i of A22 = conj(column i)
        for (int r = blockIdx.x; r < m; r += gridDim.x) {
            const double2 *col = C + (size_t)(j + 1 + r) * n + (j + 1);
            double2 acc = make_double2(0.0, 0.0);
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                const double2 p = cmulc_d(__ldcg(&col[k]), v[k]);
                acc.x += p.x;
                acc.y += p.y;
            }
            acc = block_sum<double2>(acc, red);
            if (threadIdx.x == 0) xg[r] = cmul_d(t, acc);
        }
        grid_barrier(gb, err);
        // --- w = x + alpha v, alpha = -1/2 tau (x^H v)
        double2 xv = make_double2(0.0, 0.0);
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const double2 p = cmulc_d(__ldcg(&xg[i]), v[i]);
            xv.x += p.x;
            xv.y += p.y;
        }
        xv = block_sum<double2>(xv, red);
        const double2 al = cmul_d(make_double2(-0.5 * t.x, -0.5 * t.y), xv);
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const double2 p = cmul_d(al, v[i]);
            const double2 xi = __ldcg(&xg[i]);
            w[i] = make_double2(xi.x + p.x, xi.y + p.y);
        }
        __syncthreads();
        // --- A22 -= v w^H + w v^H on owned columns
        for (int c = blockIdx.x; c < m; c += gridDim.x) {
            double2 *col = C + (size_t)(j + 1 + c) * n + (j + 1);
            const double2 wc = make_double2(w[c].x, -w[c].y), vc = make_double2(v[c].x, -v[c].y);
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const double2 a = cmul_d(v[i], wc), b = cmul_d(w[i], vc);
                col[i].x -= a.x + b.x;
                col[i].y -= a.y + b.y;
            }
        }
        for (int i = threadIdx.x; i < m; i += blockDim.x) vprev[i] = v[i];
        prev_m = m;
        grid_barrier(gb, err);
    }
    if (n >= 2 && ((n - 2) % gridDim.x) == blockIdx.x) {
        double2 *cp = C + (size_t)(n - 2) * n + (n - 1);
        for (int i = 1 + threadIdx.x; i < prev_m; i += blockDim.x) cp[i] = vprev[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) d[n - 1] = __ldcg(&C[(size_t)(n - 1) * n + (n - 1)]).x;
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

// lowest k eigenvalues of the real symmetric tridiagonal (d, e), ascending
__global__ void k_bisect(const double *__restrict__ d, const double *__restrict__ e, int n, int k, double *__restrict__ lam,
                         double *__restrict__ nrm_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    double lo = 1e300, hi = -1e300, emax2 = 0.0;
    for (int r = 0; r < n; ++r) {
        const double rad = (r > 0 ? fabs(e[r - 1]) : 0.0) + (r < n - 1 ? fabs(e[r]) : 0.0);
        lo = fmin(lo, d[r] - rad);
        hi = fmax(hi, d[r] + rad);
        if (r < n - 1) emax2 = fmax(emax2, e[r] * e[r]);
    }
    const double nrm = fmax(fabs(lo), fabs(hi));
    const double pivmin = fmax(2.2250738585072014e-308, 2.2250738585072014e-308 * emax2) * 4.0;
    double a = lo - 1e-14 * nrm - 1e-300, b = hi + 1e-14 * nrm + 1e-300;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (a + b);
        if (mid <= a || mid >= b) break;
        if (sturm_count(d, e, n, mid, pivmin) > i)
            b = mid;
        else
            a = mid;
        if (b - a <= 2.0 * 2.220446049250313e-16 * fmax(fabs(a), fabs(b))) break;
    }
    lam[i] = 0.5 * (a + b);
    if (i == 0) *nrm_out = nrm;
}

// Solve (Tr - lam I) x = b in place (b -> x) by LU with partial pivoting.
// scratch: dd, du, du2 (n each).
__device__ void tri_solve(const double *d, const double *e, int n, double lam, double *b, double *dd, double *du,
                          double *du2) {
    for (int i = 0; i < n; ++i) {
        dd[i] = d[i] - lam;
        du[i] = (i < n - 1) ? e[i] : 0.0;
        du2[i] = 0.0;
    }
    for (int i = 0; i < n - 1; ++i) {
        const double sub = e[i];
        if (fabs(dd[i]) >= fabs(sub)) {
            if (dd[i] == 0.0) dd[i] = 1e-300;
            const double f = sub / dd[i];
            dd[i + 1] -= f * du[i];
            b[i + 1] -= f * b[i];
        } else {
            const double f = dd[i] / sub;
            const double ddi1 = dd[i + 1], dui1 = du[i + 1], bi = b[i];
            dd[i] = sub;
            const double dui = du[i];
            du[i] = ddi1;
            du2[i] = dui1;
            dd[i + 1] = dui - f * ddi1;
            du[i + 1] = -f * dui1;
            b[i] = b[i + 1];
            b[i + 1] = bi - f * b[i + 1];
        }
    }
    if (dd[n - 1] == 0.0) dd[n - 1] = 1e-300;
    b[n - 1] /= dd[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / dd[n - 2];
    for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / dd[i];
}

// One warp per cluster of near-degenerate eigenvalues (gap <= ortol):
// inverse iteration for each member, re-orthogonalised against the earlier
// members of its cluster.  Z: n x k real (column-major).  work: 3n per warp.
__global__ void k_invit(const double *__restrict__ d, const double *__restrict__ e, int n, int k,
                        const double *__restrict__ lam, const double *__restrict__ nrmp, double reltol,
                        double *__restrict__ Z, double *__restrict__ work) {
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wid >= k) return;
    const double nrm = *nrmp;
    const double ortol = reltol * nrm;
    const double eps = 2.220446049250313e-16;
    // a warp owns eigenvalue wid only if it starts a cluster
    if (wid > 0 && lam[wid] - lam[wid - 1] <= ortol) return;
    double *dd = work + (size_t)wid * 3 * n, *du = dd + n, *du2 = du + n;
    int end = wid + 1;
    while (end < k && lam[end] - lam[end - 1] <= ortol) ++end;
    double lprev = 0.0;
    for (int i = wid; i < end; ++i) {
        double li = lam[i];
        if (i > wid && li - lprev < 10.0 * eps * nrm) li = lprev + 10.0 * eps * nrm;  // separate degenerate shifts
        lprev = li;
        double *x = Z + (size_t)i * n;
        // deterministic pseudo-random start
        for (int r = lane; r < n; r += 32) {
            unsigned int h = (unsigned int)(r * 2654435761u) ^ (unsigned int)(i * 2246822519u + 12345u);
            h ^= h >> 15;
            h *= 2246822519u;
            h ^= h >> 13;
            x[r] = ((double)(h & 0xFFFFFF) / 16777216.0) - 0.5;
        }
        __syncwarp();
        for (int it = 0; it < 4; ++it) {
            if (lane == 0) tri_solve(d, e, n, li, x, dd, du, du2);
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
    }
}

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
           + (size_t)n * sizeof(double2)              // xg
           + (size_t)(3 * n) * sizeof(double)         // d, e, lam
           + (size_t)n * sizeof(double2)              // tau
           + (size_t)n * k * sizeof(double)           // Ztr
           + (size_t)k * 3 * n * sizeof(double)       // inverse-iteration scratch
           + (size_t)n * k * sizeof(double2)          // Z
           + 16 * 256;                                // barrier, status, norm + 256-byte rounding of 13 pieces
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
    double2 *xg = (double2 *)take(n * sizeof(double2));
    double *d = (double *)take(n * sizeof(double));
    double *e = (double *)take(n * sizeof(double));
    double *lam = (double *)take(n * sizeof(double));
    double2 *tau = (double2 *)take(n * sizeof(double2));
    double *Zt = (double *)take((size_t)n * k * sizeof(double));
    double *iw = (double *)take((size_t)k * 3 * n * sizeof(double));
    double2 *Z = (double2 *)take((size_t)n * k * sizeof(double2));
    GridBar *gb = (GridBar *)take(sizeof(GridBar));
    int *err = (int *)take(sizeof(int) * 4);
    double *nrm = (double *)take(sizeof(double));
    cudaError_t e_;
    if ((e_ = cudaMemsetAsync(gb, 0, sizeof(GridBar), st)) != cudaSuccess) return e_;
    if ((e_ = cudaMemsetAsync(err, 0, sizeof(int) * 4, st)) != cudaSuccess) return e_;
    const int nb = blocks_for(nn);
    k_herm_upper<<<nb, 256, 0, st>>>(T, n);
    double2 *Cm = T;
    if (G) {
        k_herm_upper<<<nb, 256, 0, st>>>(G, n);
        int nblk = 0;
        if ((e_ = coop_blocks((const void *)k_chol, 0, &nblk)) != cudaSuccess) return e_;
        int *info = err + 1;
        void *args[] = {(void *)&G, (void *)&n, (void *)&gb, (void *)&err, (void *)&info};
        if ((e_ = cudaLaunchCooperativeKernel((const void *)k_chol, nblk, COOP_THREADS, args, 0, st)) != cudaSuccess)
            return e_;
        k_trinv_lower<<<(n + 7) / 8, 256, 0, st>>>(G, Linv, n);
        // C = Linv T Linv^H
        if ((e_ = gemm_nn<double>(n, n, n, Linv, n, T, n, M1, n, 0, st)) != cudaSuccess) return e_;
        k_conj_transpose<<<nb, 256, 0, st>>>(Linv, G, n);  // G no longer needed: holds Linv^H
        if ((e_ = gemm_nn<double>(n, n, n, M1, n, G, n, T, n, 0, st)) != cudaSuccess) return e_;
        k_herm_upper<<<nb, 256, 0, st>>>(T, n);
    }
    {
        const size_t smem = (size_t)(3 * n + 32) * sizeof(double2);
        int nblk = 0;
        if ((e_ = coop_blocks((const void *)k_tridiag, smem, &nblk)) != cudaSuccess) return e_;
        if ((e_ = cudaMemsetAsync(gb, 0, sizeof(GridBar), st)) != cudaSuccess) return e_;
        void *args[] = {(void *)&Cm, (void *)&n, (void *)&d, (void *)&e, (void *)&tau, (void *)&xg, (void *)&gb, (void *)&err};
        if ((e_ = cudaLaunchCooperativeKernel((const void *)k_tridiag, nblk, COOP_THREADS, args, smem, st)) != cudaSuccess)
            return e_;
    }
    k_bisect<<<(k + 127) / 128, 128, 0, st>>>(d, e, n, k, lam, nrm);
    if ((e_ = cudaMemcpyAsync(lam_out, lam, k * sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e_;
    if (S) {
        k_invit<<<(k + 7) / 8, 256, 0, st>>>(d, e, n, k, lam, nrm, 1e-7, Zt, iw);
        const size_t smem = (size_t)(n + 32) * sizeof(double2);
        if (smem > 48 * 1024 &&
            (e_ = cudaFuncSetAttribute((const void *)k_backtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
            return e_;
        k_backtr<<<k, 256, smem, st>>>(Cm, tau, n, Zt, G ? Z : S);
        if (G) {
            // S = Linv^H Z  (Linv^H sits in G)
            if ((e_ = gemm_nn<double>(n, k, n, G, n, Z, n, S, n, 0, st)) != cudaSuccess) return e_;
        }
    }
    if ((e_ = cudaGetLastError()) != cudaSuccess) return e_;
    // status: [0] barrier expiry, [1] Cholesky breakdown column (1-based)
    return cudaMemcpyAsync(d_status, err, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

cudaError_t chol_inverse_upper(double2 *C, int n, double2 *Rinv, void *work, int *d_status, cudaStream_t st) {
    unsigned char *p = (unsigned char *)work;
    double2 *Linv = (double2 *)p;
    p += (((size_t)n * n * sizeof(double2)) + 255) & ~(size_t)255;
    GridBar *gb = (GridBar *)p;
    p += 256;
    int *err = (int *)p;
    cudaError_t e_;
    if ((e_ = cudaMemsetAsync(gb, 0, sizeof(GridBar), st)) != cudaSuccess) return e_;
    if ((e_ = cudaMemsetAsync(err, 0, sizeof(int) * 4, st)) != cudaSuccess) return e_;
    const int nb = blocks_for((size_t)n * n);
    k_herm_upper<<<nb, 256, 0, st>>>(C, n);
    int nblk = 0;
    if ((e_ = coop_blocks((const void *)k_chol, 0, &nblk)) != cudaSuccess) return e_;
    int *info = err + 1;
    void *args[] = {(void *)&C, (void *)&n, (void *)&gb, (void *)&err, (void *)&info};
    if ((e_ = cudaLaunchCooperativeKernel((const void *)k_chol, nblk, COOP_THREADS, args, 0, st)) != cudaSuccess) return e_;
    k_trinv_lower<<<(n + 7) / 8, 256, 0, st>>>(C, Linv, n);
    k_conj_transpose<<<nb, 256, 0, st>>>(Linv, Rinv, n);
    if ((e_ = cudaGetLastError()) != cudaSuccess) return e_;
    return cudaMemcpyAsync(d_status, err, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

}  // namespace pwk
