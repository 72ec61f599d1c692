// pw_lobpcg_multi: diag_LOBPCG! (diag_LOBPCG.jl:51-225, the FP64 path's step
// order) advancing the blocks of many k-points together, for small blocks
// (3 nb <= 48): every step is one launch for all k-points -- op_H through
// pw_apply_multi, the Rayleigh-Ritz Grams and rotations as batched
// CUDA-core kernels with FP64 accumulation (the k-point's G+k range split
// over several CTAs), Kprec, and the small FP64 Cholesky / Hermitian
// eigenproblems one CTA per k-point in shared memory (cyclic Jacobi with
// round-robin pair ordering).  The host reads all Ritz values once per
// iteration; a k-point whose convergence test (|lambda - lambda_old| < tol
// for nconv values) holds is left alone from then on, as the per-k-point
// solver stops there.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/pwb200.h"
#include "pw_launch.h"

int pwk_fail(pw_ctx *c, int code, const char *msg);
int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out);
cudaStream_t pwk_stream(pw_ctx *c);
int pwk_ngw(const pw_ctx *c, int ik);
int pwk_device(const pw_ctx *c);
int pwk_nkpt(const pw_ctx *c);
void pwk_count_launches(pw_ctx *c, int n);
const double *pwk_gk2(const pw_ctx *c, int ik);

namespace {

constexpr int NMAX = 48;          // largest small matrix (3 nb)
constexpr int SS = NMAX * NMAX;   // stride of one small matrix per k-point
constexpr int GROWS = 16;         // G+k rows per shared-memory chunk of the Gram

struct BkDesc {
    int ngw;
    int active;
    size_t q_off;   // element offset of the k-point in the 3-block buffers (Q, HQ)
    size_t t_off;   // ... in the 2-block buffers
    const double *gk2;
};

// a block of nb-column groups in a batched buffer: base + (3 ? q_off : t_off) + blk * nb * ngw
struct BRef {
    void *base;
    int three;
    int blk;
};

template <typename C>
__device__ __forceinline__ C *bptr(const BRef &r, const BkDesc &d, int nb) {
    return reinterpret_cast<C *>(r.base) + (r.three ? d.q_off : d.t_off) + (size_t)r.blk * nb * d.ngw;
}
template <typename C> __device__ __forceinline__ double2 to_d(C v) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ double2 cm(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cmc(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }

// partial C_k = A_k^H B_k over the G+k rows of split s: part[(k * S + s) * m * n + i + m * j]
template <typename C>
__global__ void __launch_bounds__(256) bk_gram(const BkDesc *__restrict__ ds, int nb, int m, int n, BRef A, BRef B,
                                              int S, double2 *__restrict__ part) {
    __shared__ double2 As[GROWS][NMAX + 1], Bs[GROWS][NMAX + 1];
    const int k = blockIdx.x, s = blockIdx.y;
    const BkDesc d = ds[k];
    if (!d.active) return;
    const C *a = bptr<C>(A, d, nb), *b = bptr<C>(B, d, nb);
    const int per = (d.ngw + S - 1) / S, g0 = s * per, g1 = min(d.ngw, g0 + per);
    constexpr int QMAX = (NMAX * NMAX + 255) / 256;
    double2 acc[QMAX];
#pragma unroll
    for (int t = 0; t < QMAX; ++t) acc[t] = make_double2(0.0, 0.0);
    for (int c0 = g0; c0 < g1; c0 += GROWS) {
        const int rows = min(GROWS, g1 - c0);
        for (int q = threadIdx.x; q < GROWS * m; q += blockDim.x) {
            const int r = q % GROWS, i = q / GROWS;
            As[r][i] = r < rows ? to_d(a[(size_t)i * d.ngw + c0 + r]) : make_double2(0.0, 0.0);
        }
        for (int q = threadIdx.x; q < GROWS * n; q += blockDim.x) {
            const int r = q % GROWS, j = q / GROWS;
            Bs[r][j] = r < rows ? to_d(b[(size_t)j * d.ngw + c0 + r]) : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < QMAX; ++t) {
            const int q = threadIdx.x + 256 * t;
            if (q < m * n) {
                const int i = q % m, j = q / m;
                double2 v = acc[t];
                for (int r = 0; r < GROWS; ++r) {
                    const double2 p = cmc(As[r][i], Bs[r][j]);
                    v.x += p.x;
                    v.y += p.y;
                }
                acc[t] = v;
            }
        }
        __syncthreads();
    }
    double2 *out = part + ((size_t)k * S + s) * m * n;
#pragma unroll
    for (int t = 0; t < QMAX; ++t) {
        const int q = threadIdx.x + 256 * t;
        if (q < m * n) out[q] = acc[t];
    }
}

// C_k (small, stride SS, ld m) = sum over splits
__global__ void bk_gram_reduce(const BkDesc *__restrict__ ds, int m, int n, int S, const double2 *__restrict__ part,
                               double2 *__restrict__ Csm) {
    const int k = blockIdx.x;
    if (!ds[k].active) return;
    for (int q = threadIdx.x; q < m * n; q += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int s = 0; s < S; ++s) {
            const double2 p = part[((size_t)k * S + s) * m * n + q];
            v.x += p.x;
            v.y += p.y;
        }
        Csm[(size_t)k * SS + q] = v;
    }
}

// Cout_k (ngw x n) (+)= A_k (ngw x m) U_k (m x n; small matrix of k, offset uoff, ld ldu)
template <typename C>
__global__ void __launch_bounds__(256) bk_rot(const BkDesc *__restrict__ ds, int nb, int m, int n, BRef A,
                                             const double2 *__restrict__ Usm, int uoff, int ldu, BRef Cout, int acc) {
    __shared__ double2 Us[NMAX * 16];
    const int k = blockIdx.x;
    const BkDesc d = ds[k];
    if (!d.active) return;
    const double2 *U = Usm + (size_t)k * SS + uoff;
    for (int q = threadIdx.x; q < m * n; q += blockDim.x) Us[q] = U[(q % m) + (size_t)(q / m) * ldu];
    __syncthreads();
    const C *a = bptr<C>(A, d, nb);
    C *c = bptr<C>(Cout, d, nb);
    for (int g = blockIdx.y * blockDim.x + threadIdx.x; g < d.ngw; g += gridDim.y * blockDim.x) {
        double2 v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = make_double2(0.0, 0.0);
        for (int i = 0; i < m; ++i) {
            const double2 x = to_d(a[(size_t)i * d.ngw + g]);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (j < n) {
                    const double2 p = cm(x, Us[i + m * j]);
                    v[j].x += p.x;
                    v[j].y += p.y;
                }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (j < n) {
                C *o = c + (size_t)j * d.ngw + g;
                if (acc) {
                    v[j].x += (double)o->x;
                    v[j].y += (double)o->y;
                }
                o->x = (decltype(o->x))v[j].x;
                o->y = (decltype(o->y))v[j].y;
            }
    }
}

// dst = src (ncols columns); kprec != 0: dst = src / (1 + |G+k|^2) (Kprec.jl:30-44)
template <typename C>
__global__ void bk_copy(const BkDesc *__restrict__ ds, int nb, int ncols, BRef Src, BRef Dst, int kprec) {
    const int k = blockIdx.x;
    const BkDesc d = ds[k];
    if (!d.active) return;
    const C *s = bptr<C>(Src, d, nb);
    C *t = bptr<C>(Dst, d, nb);
    const size_t tot = (size_t)ncols * d.ngw;
    for (size_t q = blockIdx.y * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.y * blockDim.x) {
        C v = s[q];
        if (kprec) {
            const double f = 1.0 / (1.0 + d.gk2[q % d.ngw]);
            v.x = (decltype(v.x))(v.x * f);
            v.y = (decltype(v.y))(v.y * f);
        }
        t[q] = v;
    }
}

// copies between the user's blocks (pointer per k, ld per k) and a batched block
template <typename C>
__global__ void bk_user(const BkDesc *__restrict__ ds, int nb, C *const *__restrict__ user, const int64_t *__restrict__ uld,
                        BRef Blk, int to_user) {
    const int k = blockIdx.x;
    const BkDesc d = ds[k];
    C *b = bptr<C>(Blk, d, nb);
    C *u = user[k];
    const size_t tot = (size_t)nb * d.ngw;
    for (size_t q = blockIdx.y * (size_t)blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.y * blockDim.x) {
        const size_t j = q / d.ngw, g = q - j * d.ngw;
        if (to_user)
            u[j * uld[k] + g] = b[q];
        else
            b[q] = u[j * uld[k] + g];
    }
}

// ---------------------------------------------- small FP64 dense (one CTA per k)
// Hermitian matrices of order n <= NMAX held column-major in shared memory.

// Hermitian part from the upper triangle, real diagonal (Hermitian(A) of Julia)
__device__ void herm_from_upper(double2 *A, int n) {
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q % n, j = q / n;
        if (i > j) A[q] = make_double2(A[j + n * i].x, -A[j + n * i].y);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) A[i + n * i].y = 0.0;
    __syncthreads();
}

// lower Cholesky factor in place (upper triangle left as is); returns 0 or
// the 1-based failing column (not positive definite)
__device__ int chol_lower(double2 *A, int n, int *fail) {
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) {
            const double djj = A[j + n * j].x;
            if (!(djj > 0.0) && *fail == 0) *fail = j + 1;
            A[j + n * j] = make_double2(djj > 0.0 ? sqrt(djj) : 1.0, 0.0);
        }
        __syncthreads();
        const double inv = 1.0 / A[j + n * j].x;
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            A[i + n * j].x *= inv;
            A[i + n * j].y *= inv;
        }
        __syncthreads();
        // trailing update A[i][l] -= L[i][j] conj(L[l][j]) for l <= i, l > j
        for (int q = threadIdx.x; q < (n - j - 1) * (n - j - 1); q += blockDim.x) {
            const int i = j + 1 + q % (n - j - 1), l = j + 1 + q / (n - j - 1);
            if (l <= i) {
                const double2 p = cmc(A[l + n * j], A[i + n * j]);   // conj(L[l][j]) L[i][j]
                A[i + n * l].x -= p.x;
                A[i + n * l].y -= p.y;
            }
        }
        __syncthreads();
    }
    return *fail;
}

// Li = L^-1 (lower triangular) by columns: Li[:, c] solves L x = e_c
__device__ void tri_inverse_lower(const double2 *L, double2 *Li, int n) {
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) Li[q] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        for (int i = c; i < n; ++i) {
            double2 s = make_double2(i == c ? 1.0 : 0.0, 0.0);
            for (int t = c; t < i; ++t) {
                const double2 p = cm(L[i + n * t], Li[t + n * c]);
                s.x -= p.x;
                s.y -= p.y;
            }
            const double di = 1.0 / L[i + n * i].x;
            Li[i + n * c] = make_double2(s.x * di, s.y * di);
        }
    }
    __syncthreads();
}

// out = X Y (n x n), all column-major in shared memory; conjX / conjY: use X^H / Y^H
__device__ void small_mm(const double2 *X, const double2 *Y, double2 *out, int n, bool cx, bool cy) {
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q % n, j = q / n;
        double2 s = make_double2(0.0, 0.0);
        for (int t = 0; t < n; ++t) {
            double2 x = cx ? make_double2(X[t + n * i].x, -X[t + n * i].y) : X[i + n * t];
            double2 y = cy ? make_double2(Y[j + n * t].x, -Y[j + n * t].y) : Y[t + n * j];
            const double2 p = cm(x, y);
            s.x += p.x;
            s.y += p.y;
        }
        out[q] = s;
    }
    __syncthreads();
}

// Hermitian Jacobi: A (n x n) diagonalised in place, V (if non-null) := V J
// accumulated.  Round-robin pairs, n rounded up to even (index n is a dummy).
__device__ void jacobi(double2 *A, double2 *V, int n, double2 *rot /* [NMAX/2+1] c, s */, double *phi, int *pp, int *pq,
                       double *red) {
    const int ne = n + (n & 1);
    for (int sweep = 0; sweep < 40; ++sweep) {
        // off-diagonal and total norms
        double off = 0.0, tot = 0.0;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q % n, j = q / n;
            const double v = A[q].x * A[q].x + A[q].y * A[q].y;
            tot += v;
            if (i != j) off += v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((threadIdx.x & 31) == 0) {
            red[2 * (threadIdx.x >> 5)] = off;
            red[2 * (threadIdx.x >> 5) + 1] = tot;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                a += red[2 * w];
                b += red[2 * w + 1];
            }
            red[64] = a;
            red[65] = b;
        }
        __syncthreads();
        if (!(red[64] > 1e-26 * red[65]) || n < 2) break;   // relative off-diagonal norm 1e-13
        __syncthreads();
        for (int step = 0; step < ne - 1; ++step) {
            // pairs of this step of the round-robin ordering: position 0 fixed, the others rotate
            const int np = ne / 2;
            for (int t = threadIdx.x; t < np; t += blockDim.x) {
                auto at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + step) % (ne - 1); };
                int p = at(t), q = at(ne - 1 - t);
                if (p > q) {
                    const int x = p;
                    p = q;
                    q = x;
                }
                pp[t] = p;
                pq[t] = q;
                double c = 1.0, sn = 0.0, ph = 0.0;
                if (q < n) {
                    const double2 b = A[p + n * q];
                    const double ab = sqrt(b.x * b.x + b.y * b.y);
                    if (ab > 1e-300) {
                        const double a = A[p + n * p].x, dd = A[q + n * q].x;
                        const double tau = (dd - a) / (2.0 * ab);
                        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        sn = tt * c;
                        ph = atan2(b.y, b.x);
                    }
                }
                rot[t] = make_double2(c, sn);
                phi[t] = ph;
            }
            __syncthreads();
            // columns: A_p <- c A_p - s e^{-i phi} A_q ; A_q <- s A_p + c e^{-i phi} A_q (and V alike)
            for (int q2 = threadIdx.x; q2 < np * n; q2 += blockDim.x) {
                const int t = q2 / n, i = q2 % n;
                const int p = pp[t], q = pq[t];
                if (q >= n) continue;
                const double c = rot[t].x, s = rot[t].y;
                const double2 e = make_double2(cos(phi[t]), -sin(phi[t]));   // e^{-i phi}
                for (int mtx = 0; mtx < (V ? 2 : 1); ++mtx) {
                    double2 *M = mtx ? V : A;
                    const double2 xp = M[i + n * p], xq = cm(M[i + n * q], e);
                    M[i + n * p] = make_double2(c * xp.x - s * xq.x, c * xp.y - s * xq.y);
                    M[i + n * q] = make_double2(s * xp.x + c * xq.x, s * xp.y + c * xq.y);
                }
            }
            __syncthreads();
            // rows: row_p <- c row_p - s e^{i phi} row_q ; row_q <- s row_p + c e^{i phi} row_q
            for (int q2 = threadIdx.x; q2 < np * n; q2 += blockDim.x) {
                const int t = q2 / n, j = q2 % n;
                const int p = pp[t], q = pq[t];
                if (q >= n) continue;
                const double c = rot[t].x, s = rot[t].y;
                const double2 e = make_double2(cos(phi[t]), sin(phi[t]));     // e^{+i phi}
                const double2 xp = A[p + n * j], xq = cm(A[q + n * j], e);
                A[p + n * j] = make_double2(c * xp.x - s * xq.x, c * xp.y - s * xq.y);
                A[q + n * j] = make_double2(s * xp.x + c * xq.x, s * xp.y + c * xq.y);
            }
            __syncthreads();
        }
    }
}

struct SmallWork {
    double2 rot[NMAX / 2 + 1];
    double phi[NMAX / 2 + 1];
    int pp[NMAX / 2 + 1], pq[NMAX / 2 + 1];
    double red[72];
    int order[NMAX];
    int fail;
};

// ascending order of the diagonal of A into order[] (one thread; n <= 48)
__device__ void sort_diag(const double2 *A, int n, int *order) {
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) order[i] = i;
        for (int i = 1; i < n; ++i) {
            const int v = order[i];
            const double key = A[v + n * v].x;
            int j = i - 1;
            while (j >= 0 && A[order[j] + n * order[j]].x > key) {
                order[j + 1] = order[j];
                --j;
            }
            order[j + 1] = v;
        }
    }
    __syncthreads();
}

// mode 0: eigenvalues of Hermitian(M) (order n) into lam[k*lstride ..];
// mode 1: lowest nev pairs of (Hermitian(T), Hermitian(G)), vectors (n x nev, ld n) into S;
// mode 2: Rinv = R^-1 with Hermitian(C) = R^H R (into S, n x n);
// mode 3: all pairs of Hermitian(T) (standard), vectors into S.
// status[k] = 1-based failing Cholesky column, 0 on success.
__global__ void __launch_bounds__(256) bk_small(const BkDesc *__restrict__ ds, int mode, int n, int nev,
                                                const double2 *__restrict__ Tsm, const double2 *__restrict__ Gsm,
                                                double *__restrict__ lam, int lstride, double2 *__restrict__ Ssm,
                                                int *__restrict__ status) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *A = reinterpret_cast<double2 *>(sm);
    double2 *B = A + n * n;
    double2 *Cm = B + n * n;
    double2 *V = Cm + n * n;
    __shared__ SmallWork w;
    const int k = blockIdx.x;
    if (!ds[k].active) return;
    if (threadIdx.x == 0) w.fail = 0;
    const double2 *T = Tsm + (size_t)k * SS;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) A[q] = T[q];
    __syncthreads();
    herm_from_upper(A, n);
    if (mode == 2) {
        chol_lower(A, n, &w.fail);           // C = L L^H, R = L^H
        tri_inverse_lower(A, B, n);          // B = L^-1 ; R^-1 = (L^-1)^H
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q % n, j = q / n;
            Ssm[(size_t)k * SS + q] = make_double2(B[j + n * i].x, -B[j + n * i].y);
        }
        if (threadIdx.x == 0) status[k] = w.fail;
        return;
    }
    if (mode == 1) {
        const double2 *G = Gsm + (size_t)k * SS;
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) B[q] = G[q];
        __syncthreads();
        herm_from_upper(B, n);
        chol_lower(B, n, &w.fail);
        tri_inverse_lower(B, Cm, n);         // Cm = L^-1
        small_mm(Cm, A, V, n, false, false); // V = L^-1 T
        small_mm(V, Cm, A, n, false, true);  // A = L^-1 T L^-H
        herm_from_upper(A, n);
    }
    const bool vec = mode != 0;
    if (vec) {
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) V[q] = make_double2((q % n) == (q / n) ? 1.0 : 0.0, 0.0);
        __syncthreads();
    }
    jacobi(A, vec ? V : nullptr, n, w.rot, w.phi, w.pp, w.pq, w.red);
    sort_diag(A, n, w.order);
    const int ne = mode == 1 ? nev : n;
    for (int i = threadIdx.x; i < ne; i += blockDim.x) lam[(size_t)k * lstride + i] = A[w.order[i] + n * w.order[i]].x;
    if (mode == 3) {
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
            const int i = q % n, j = q / n;
            Ssm[(size_t)k * SS + q] = V[i + n * w.order[j]];
        }
    }
    if (mode == 1) {
        // S = L^-H V[:, order[0..nev)]
        for (int q = threadIdx.x; q < n * nev; q += blockDim.x) {
            const int i = q % n, j = q / n;
            double2 s = make_double2(0.0, 0.0);
            for (int t = i; t < n; ++t) {
                const double2 li = make_double2(Cm[t + n * i].x, -Cm[t + n * i].y);   // (L^-H)[i][t] = conj(L^-1[t][i])
                const double2 p = cm(li, V[t + n * w.order[j]]);
                s.x += p.x;
                s.y += p.y;
            }
            Ssm[(size_t)k * SS + q] = s;
        }
        if (threadIdx.x == 0) status[k] = w.fail;
    }
}

// small matrices: out = -in (n x n); or (in + in^H)/2 written to both triangles
__global__ void bk_small_ew(const BkDesc *__restrict__ ds, int n, const double2 *__restrict__ in, double2 *__restrict__ out,
                            int mode) {
    const int k = blockIdx.x;
    if (!ds[k].active) return;
    const double2 *a = in + (size_t)k * SS;
    double2 *b = out + (size_t)k * SS;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int i = q % n, j = q / n;
        if (mode == 0)
            b[q] = make_double2(-a[q].x, -a[q].y);
        else
            b[q] = make_double2(0.5 * (a[q].x + a[j + n * i].x), 0.5 * (a[q].y - a[j + n * i].y));
    }
}

#define CKM(c, x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, #x " failed"); \
    } while (0)
#define RKM(x)                        \
    do {                              \
        int s_ = (x);                 \
        if (s_ != PW_OK) return s_;   \
    } while (0)

template <typename C>
struct Batch {
    pw_ctx *c;
    cudaStream_t st;
    int nk, nb, S, ngw_max;
    const BkDesc *d_desc;
    double2 *part;
    std::vector<BkDesc> desc;

    int gram(int m, int n, BRef A, BRef B, double2 *Csm) {
        bk_gram<C><<<dim3(nk, S), 256, 0, st>>>(d_desc, nb, m, n, A, B, S, part);
        bk_gram_reduce<<<nk, 256, 0, st>>>(d_desc, m, n, S, part, Csm);
        CKM(c, cudaGetLastError());
        pwk_count_launches(c, 2);
        return PW_OK;
    }
    int rot(int m, int n, BRef A, const double2 *Usm, int uoff, int ldu, BRef Cout, int acc) {
        const int gy = std::max(1, std::min(64, (ngw_max + 255) / 256));
        bk_rot<C><<<dim3(nk, gy), 256, 0, st>>>(d_desc, nb, m, n, A, Usm, uoff, ldu, Cout, acc);
        CKM(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        return PW_OK;
    }
    int copy(int ncols, BRef Src, BRef Dst, int kprec) {
        const int gy = std::max(1, std::min(64, (ncols * ngw_max + 255) / 256));
        bk_copy<C><<<dim3(nk, gy), 256, 0, st>>>(d_desc, nb, ncols, Src, Dst, kprec);
        CKM(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        return PW_OK;
    }
    int small(int mode, int n, int nev, const double2 *T, const double2 *G, double *lam, int lstride, double2 *S,
              int *status) {
        const size_t smem = 4 * (size_t)n * n * sizeof(double2);
        if (smem > 48 * 1024)
            CKM(c, cudaFuncSetAttribute((const void *)bk_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bk_small<<<nk, 256, smem, st>>>(d_desc, mode, n, nev, T, G, lam, lstride, S, status);
        CKM(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        return PW_OK;
    }
    int ew(int n, const double2 *in, double2 *out, int mode) {
        bk_small_ew<<<nk, 256, 0, st>>>(d_desc, n, in, out, mode);
        CKM(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        return PW_OK;
    }
    // host copy of the per-k status words; PW_ERR_NOT_POSDEF when any is set
    int check(int *d_status, std::vector<int> &h) {
        CKM(c, cudaMemcpyAsync(h.data(), d_status, nk * sizeof(int), cudaMemcpyDeviceToHost, st));
        CKM(c, cudaStreamSynchronize(st));
        for (int k = 0; k < nk; ++k)
            if (desc[k].active && h[k]) return pwk_fail(c, PW_ERR_NOT_POSDEF, "cholesky(Hermitian(C)) failed: C not positive definite");
        return PW_OK;
    }
};

template <typename C>
int lobpcg_multi(pw_ctx *c, int nk, const int *iks, int ispin, int dtype, void *const *X, const int64_t *ld, int nb,
                 double tol, int nitermax, int nconv_target, double *evals, int *niter_out) {
    Batch<C> B;
    B.c = c;
    B.st = pwk_stream(c);
    B.nk = nk;
    B.nb = nb;
    B.desc.resize(nk);
    size_t q_tot = 0, t_tot = 0;
    int ngw_max = 0;
    for (int k = 0; k < nk; ++k) {
        const int ngw = pwk_ngw(c, iks[k]);
        B.desc[k] = BkDesc{ngw, 1, q_tot, t_tot, pwk_gk2(c, iks[k])};
        q_tot += 3 * (size_t)nb * ngw;
        t_tot += 2 * (size_t)nb * ngw;
        ngw_max = std::max(ngw_max, ngw);
    }
    B.ngw_max = ngw_max;
    B.S = std::max(1, std::min(16, (2 * 148 + nk - 1) / nk));
    const int n3 = 3 * nb;
    char *Q, *HQ, *T1, *T2, *small;
    void *misc;
    RKM(pwk_scratch(c, pwk::SL_LOB_Q, q_tot * sizeof(C), (void **)&Q));
    RKM(pwk_scratch(c, pwk::SL_LOB_HQ, q_tot * sizeof(C), (void **)&HQ));
    RKM(pwk_scratch(c, pwk::SL_LOB_TMP1, t_tot * sizeof(C), (void **)&T1));
    RKM(pwk_scratch(c, pwk::SL_LOB_TMP2, t_tot * sizeof(C), (void **)&T2));
    constexpr int NSM = 8;   // XHX, M1, Rinv, T3, G3, S3, Sfin, spare
    RKM(pwk_scratch(c, pwk::SL_LOB_SMALL, (size_t)NSM * nk * SS * sizeof(double2), (void **)&small));
    const size_t part_b = (size_t)nk * B.S * SS * sizeof(double2);
    const size_t desc_b = ((nk * sizeof(BkDesc)) + 255) & ~(size_t)255;
    const size_t lam_b = (((size_t)nk * NMAX * sizeof(double)) + 255) & ~(size_t)255;
    const size_t ptr_b = ((nk * (sizeof(void *) + sizeof(int64_t) + sizeof(int))) + 255) & ~(size_t)255;
    RKM(pwk_scratch(c, pwk::SL_LOB_EIGW, part_b + desc_b + lam_b + ptr_b, &misc));
    B.part = (double2 *)misc;
    BkDesc *d_desc = (BkDesc *)((char *)misc + part_b);
    double *d_lam = (double *)((char *)d_desc + desc_b);
    char *d_ptrs = (char *)d_lam + lam_b;
    C **d_user = (C **)d_ptrs;
    int64_t *d_uld = (int64_t *)(d_ptrs + nk * sizeof(void *));
    int *d_status = (int *)(d_uld + nk);
    B.d_desc = d_desc;
    double2 *XHX = (double2 *)small, *M1 = XHX + (size_t)nk * SS, *Rinv = M1 + (size_t)nk * SS;
    double2 *T3 = Rinv + (size_t)nk * SS, *G3 = T3 + (size_t)nk * SS, *S3 = G3 + (size_t)nk * SS;
    double2 *Sfin = S3 + (size_t)nk * SS;
    cudaStream_t st = B.st;
    auto upload_desc = [&]() -> int {
        CKM(c, cudaMemcpyAsync(d_desc, B.desc.data(), nk * sizeof(BkDesc), cudaMemcpyHostToDevice, st));
        return PW_OK;
    };
    RKM(upload_desc());
    {
        std::vector<void *> up(X, X + nk);
        CKM(c, cudaMemcpyAsync(d_user, up.data(), nk * sizeof(void *), cudaMemcpyHostToDevice, st));
        CKM(c, cudaMemcpyAsync(d_uld, ld, nk * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CKM(c, cudaStreamSynchronize(st));
    }
    const BRef Xq{Q, 1, 0}, Wq{Q, 1, 1}, Pq{Q, 1, 2}, HXq{HQ, 1, 0}, HWq{HQ, 1, 1}, HPq{HQ, 1, 2};
    const BRef Qall{Q, 1, 0}, HQall{HQ, 1, 0}, Xn{T1, 0, 0}, Pn{T1, 0, 1}, HXn{T2, 0, 0}, HPn{T2, 0, 1};
    const int uy = std::max(1, std::min(64, (nb * ngw_max + 255) / 256));
    bk_user<C><<<dim3(nk, uy), 256, 0, st>>>(d_desc, nb, d_user, d_uld, Xq, 0);
    CKM(c, cudaGetLastError());
    // op_H on the Q / HQ blocks of the active k-points
    std::vector<void *> pin(nk), pout(nk);
    std::vector<int64_t> pld(nk);
    std::vector<int> pnb(nk, nb), pik(nk);
    auto apply = [&](int blk) -> int {
        int na = 0;
        for (int k = 0; k < nk; ++k) {
            if (!B.desc[k].active) continue;
            const size_t off = B.desc[k].q_off + (size_t)blk * nb * B.desc[k].ngw;
            pin[na] = (C *)Q + off;
            pout[na] = (C *)HQ + off;
            pld[na] = B.desc[k].ngw;
            pik[na] = iks[k];
            ++na;
        }
        if (na == 0) return PW_OK;
        return pw_apply_multi(c, na, pik.data(), ispin, dtype, pin.data(), pout.data(), pld.data(), pnb.data(), PW_OP_H);
    };
    RKM(apply(0));
    std::vector<double> ev((size_t)nk * NMAX), ev_old((size_t)nk * NMAX, 0.0);
    std::vector<int> hstat(nk);
    int it = 0, iters_done = 0;
    for (it = 1; it <= nitermax; ++it) {
        // XHX = X'HX and its eigenvalues (:85-86); convergence (:88-97)
        RKM(B.gram(nb, nb, Xq, HXq, XHX));
        RKM(B.small(0, nb, nb, XHX, nullptr, d_lam, NMAX, nullptr, d_status));
        CKM(c, cudaMemcpyAsync(ev.data(), d_lam, ev.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CKM(c, cudaStreamSynchronize(st));
        int nact = 0;
        for (int k = 0; k < nk; ++k) {
            if (!B.desc[k].active) continue;
            int nconv = 0;
            for (int i = 0; i < nb; ++i) {
                const double v = ev[(size_t)k * NMAX + i];
                if (!std::isfinite(v)) return pwk_fail(c, PW_ERR_NAN, "non-finite Ritz value in LOBPCG");
                if (std::fabs(v - ev_old[(size_t)k * NMAX + i]) < tol) ++nconv;
                ev_old[(size_t)k * NMAX + i] = v;
            }
            if (nconv >= nconv_target)
                B.desc[k].active = 0;
            else
                ++nact;
        }
        if (nact == 0) break;
        iters_done = it;
        RKM(upload_desc());
        // R = HX - X XHX; W = Kprec(R) (:92, :123)
        RKM(B.ew(nb, XHX, M1, 0));
        RKM(B.copy(nb, HXq, Wq, 0));
        RKM(B.rot(nb, nb, Xq, M1, 0, nb, Wq, 1));
        RKM(B.copy(nb, Wq, Wq, 1));
        // HW = op_H(W); C = W'W = R^H R; W = W/R; HW = HW/R (:167-174)
        RKM(apply(1));
        RKM(B.gram(nb, nb, Wq, Wq, M1));
        RKM(B.small(2, nb, nb, M1, nullptr, d_lam, NMAX, Rinv, d_status));
        RKM(B.check(d_status, hstat));
        RKM(B.rot(nb, nb, Wq, Rinv, 0, nb, Xn, 0));
        RKM(B.copy(nb, Xn, Wq, 0));
        RKM(B.rot(nb, nb, HWq, Rinv, 0, nb, Xn, 0));
        RKM(B.copy(nb, Xn, HWq, 0));
        // Rayleigh-Ritz on [X W (P)] (:176-185)
        const int nq = it > 1 ? n3 : 2 * nb;
        RKM(B.gram(nq, nq, Qall, HQall, T3));
        RKM(B.gram(nq, nq, Qall, Qall, G3));
        RKM(B.small(1, nq, nb, T3, G3, d_lam, NMAX, S3, d_status));
        RKM(B.check(d_status, hstat));
        // X = Q U, HX = HQ U (:187-189)
        RKM(B.rot(nq, nb, Qall, S3, 0, nq, Xn, 0));
        RKM(B.rot(nq, nb, HQall, S3, 0, nq, HXn, 0));
        if (nq == n3) {
            // P = [W P] U[nb:], HP = [HW HP] U[nb:]; P = P/R, HP = HP/R (:190-199)
            RKM(B.rot(2 * nb, nb, Wq, S3, nb, nq, Pn, 0));
            RKM(B.rot(2 * nb, nb, HWq, S3, nb, nq, HPn, 0));
            RKM(B.gram(nb, nb, Pn, Pn, M1));
            RKM(B.small(2, nb, nb, M1, nullptr, d_lam, NMAX, Rinv, d_status));
            RKM(B.check(d_status, hstat));
            RKM(B.rot(nb, nb, Pn, Rinv, 0, nb, Pq, 0));
            RKM(B.rot(nb, nb, HPn, Rinv, 0, nb, HPq, 0));
        } else {
            // P = W, HP = HW (:201-202)
            RKM(B.copy(nb, Wq, Pq, 0));
            RKM(B.copy(nb, HWq, HPq, 0));
        }
        RKM(B.copy(nb, Xn, Xq, 0));
        RKM(B.copy(nb, HXn, HXq, 0));
    }
    // final Rayleigh-Ritz: S = X'HX, S = (S+S')/2, X = X Q (:214-217)
    for (auto &d : B.desc) d.active = 1;
    RKM(upload_desc());
    RKM(B.gram(nb, nb, Xq, HXq, Sfin));
    RKM(B.ew(nb, Sfin, M1, 1));
    RKM(B.small(3, nb, nb, M1, nullptr, d_lam, NMAX, Sfin, d_status));
    RKM(B.rot(nb, nb, Xq, Sfin, 0, nb, Xn, 0));
    bk_user<C><<<dim3(nk, uy), 256, 0, st>>>(d_desc, nb, d_user, d_uld, Xn, 1);
    CKM(c, cudaGetLastError());
    CKM(c, cudaMemcpyAsync(ev.data(), d_lam, ev.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKM(c, cudaStreamSynchronize(st));
    for (int k = 0; k < nk; ++k)
        for (int i = 0; i < nb; ++i) evals[(size_t)k * nb + i] = ev[(size_t)k * NMAX + i];
    if (niter_out) *niter_out = iters_done;
    return PW_OK;
}

}  // namespace

extern "C" int pw_lobpcg_multi(pw_ctx *c, int nk, const int *iks, int ispin, int dtype, void *const *X, const int64_t *ld,
                               int nb, double tol, int nitermax, int nconv, double *evals, int *niter) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (nk <= 0 || !iks || !X || !ld || !evals || nb <= 0 || nitermax <= 0)
        return pwk_fail(c, PW_ERR_ARG, "bad pw_lobpcg_multi arguments");
    if (3 * nb > NMAX) return pwk_fail(c, PW_ERR_UNSUPPORTED, "pw_lobpcg_multi takes blocks of at most 16 bands");
    for (int k = 0; k < nk; ++k) {
        if (iks[k] < 0 || iks[k] >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
        if (!X[k] || ld[k] < pwk_ngw(c, iks[k]) || 3 * nb > pwk_ngw(c, iks[k]))
            return pwk_fail(c, PW_ERR_ARG, "bad block of pw_lobpcg_multi (need ld >= Ngw and 3 nb <= Ngw)");
    }
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    if (nconv <= 0) nconv = nb;
    return dtype == PW_C128 ? lobpcg_multi<double2>(c, nk, iks, ispin, dtype, X, ld, nb, tol, nitermax, nconv, evals, niter)
                            : lobpcg_multi<float2>(c, nk, iks, ispin, dtype, X, ld, nb, tol, nitermax, nconv, evals, niter);
}
