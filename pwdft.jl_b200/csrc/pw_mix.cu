// mix_pulay! (mix_pulay.jl:1-41) on the device, with the history kept in
// the context between SCF iterations.
//
// The reference keeps the last MIXDIM differences dx = x - x_old and
// df = f - f_old (f = gx - x) as the columns of X and F, shifting them left
// once full, and from iteration MIXDIM + 1 on mixes
//     x := x + beta f - (X + beta F) inv(F'F) (F'f)
// (simple mixing x + beta f before that).  Here the history is a ring of
// MIXDIM slots (slot (iter - 1) mod MIXDIM): the products F'F and F'f do not
// depend on the column order, so only the new slot's row of F'F and the whole
// F'f are formed each iteration, in one pass over the density that also
// stores dx, df, x_old and f_old.  The small solve (Gaussian elimination with
// partial pivoting, FP64, one warp) and the final update are two more
// launches; nothing returns to the host.  The KS_solve_SCF.jl:277-281 clamp
// rho >= eps() is fused into the update.
#include <cfloat>

#include "../../include/pwb200.h"
#include "pw_launch.h"

cudaStream_t pwk_stream(pw_ctx *c);
int pwk_device(const pw_ctx *c);
int pwk_fail_msg(pw_ctx *c, int code, const char *msg);
void pwk_count_launches(pw_ctx *c, int n);
void **pwk_mix_slot(pw_ctx *c);

namespace {

constexpr int MIX_MAX = 16;      // largest history the kernels hold in registers
constexpr int MIX_BLOCKS = 296;  // 2 x 148 SMs: fixed, so the partial sums reduce in a fixed order
constexpr int MIX_THREADS = 256;

struct MixState {
    int64_t n = 0;
    int dim = 0;
    double *X = nullptr, *F = nullptr;        // dim x n each (slot-major)
    double *xold = nullptr, *fold = nullptr;  // n each
    double *part = nullptr;                   // MIX_BLOCKS x 2 dim partial sums
    double *FtF = nullptr;                    // dim x dim
    double *coef = nullptr;                   // dim (0 for simple mixing)
    void *mem = nullptr;
};

// pass 1: f = gx - x, dx / df, history slot `slot`, x_old / f_old, and the
// block partials of  row[j] = df . F_j  and  rhs[j] = F_j . f  (F_slot = df)
template <int D>
__global__ void __launch_bounds__(MIX_THREADS)
k_pulay_hist(const double *__restrict__ x, const double *__restrict__ gx, double *__restrict__ X,
             double *__restrict__ F, double *__restrict__ xold, double *__restrict__ fold, int64_t n, int dim, int slot,
             int first, double *__restrict__ part) {
    double row[D], rhs[D];
#pragma unroll
    for (int j = 0; j < D; ++j) row[j] = rhs[j] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double xi = x[i], fi = gx[i] - xi;
        const double dx = first ? xi : xi - xold[i];
        const double df = first ? fi : fi - fold[i];
        X[(size_t)slot * n + i] = dx;
        F[(size_t)slot * n + i] = df;
        xold[i] = xi;
        fold[i] = fi;
#pragma unroll
        for (int j = 0; j < D; ++j) {
            if (j < dim) {
                const double Fj = j == slot ? df : F[(size_t)j * n + i];
                row[j] += df * Fj;
                rhs[j] += Fj * fi;
            }
        }
    }
    __shared__ double red[MIX_THREADS / 32][2 * D];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        double a = row[j], b = rhs[j];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            red[w][j] = a;
            red[w][D + j] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * dim) {
        const int k = threadIdx.x < dim ? threadIdx.x : D + threadIdx.x - dim;
        double s = 0.0;
        for (int q = 0; q < MIX_THREADS / 32; ++q) s += red[q][k];
        part[(size_t)blockIdx.x * 2 * dim + threadIdx.x] = s;
    }
}

// pass 2 (one warp): sums the partials in block order, updates the
// symmetric F'F with the new slot's row, and for iter > dim solves
// (F'F) c = F'f; coef = c (zeros before the Pulay steps start, or when the
// system is singular: that iteration then mixes simply)
__global__ void k_pulay_solve(const double *__restrict__ part, int nblocks, int dim, int slot, int pulay,
                              double *__restrict__ FtF, double *__restrict__ coef) {
    __shared__ double row[MIX_MAX], rhs[MIX_MAX], A[MIX_MAX][MIX_MAX + 1];
    const int lane = threadIdx.x;
    if (lane < 2 * dim) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * 2 * dim + lane];
        if (lane < dim)
            row[lane] = s;
        else
            rhs[lane - dim] = s;
    }
    __syncwarp();
    if (lane < dim) {
        FtF[(size_t)slot * dim + lane] = row[lane];
        FtF[(size_t)lane * dim + slot] = row[lane];
    }
    __syncwarp();
    if (!pulay) {
        if (lane < dim) coef[lane] = 0.0;
        return;
    }
    for (int i = lane; i < dim * dim; i += 32) A[i / dim][i % dim] = FtF[i];
    if (lane < dim) A[lane][dim] = rhs[lane];
    __syncwarp();
    bool ok = true;
    for (int k = 0; k < dim && ok; ++k) {
        // partial pivoting: row with the largest |A[r][k]|, r >= k (lane 0 decides)
        __shared__ int piv;
        if (lane == 0) {
            int p = k;
            for (int r = k + 1; r < dim; ++r)
                if (fabs(A[r][k]) > fabs(A[p][k])) p = r;
            piv = p;
        }
        __syncwarp();
        const int p = piv;
        if (!(fabs(A[p][k]) > DBL_MIN)) {
            ok = false;
            break;
        }
        if (p != k)
            for (int c = lane; c <= dim; c += 32) {
                const double t = A[k][c];
                A[k][c] = A[p][c];
                A[p][c] = t;
            }
        __syncwarp();
        const double inv = 1.0 / A[k][k];
        for (int r = k + 1 + lane; r < dim; r += 32) {
            const double m = A[r][k] * inv;
            for (int c = k; c <= dim; ++c) A[r][c] -= m * A[k][c];
        }
        __syncwarp();
    }
    if (lane == 0) {
        if (ok) {
            for (int k = dim - 1; k >= 0; --k) {
                double s = A[k][dim];
                for (int c = k + 1; c < dim; ++c) s -= A[k][c] * coef[c];
                coef[k] = s / A[k][k];
            }
        } else {
            for (int k = 0; k < dim; ++k) coef[k] = 0.0;
        }
    }
}

// pass 3: x := x + beta f - sum_j c_j (X_j + beta F_j), then x >= eps()
template <int D>
__global__ void __launch_bounds__(MIX_THREADS)
k_pulay_apply(double *__restrict__ x, const double *__restrict__ gx, const double *__restrict__ X,
              const double *__restrict__ F, const double *__restrict__ coef, int64_t n, int dim, double beta,
              int clamp) {
    double c[D];
#pragma unroll
    for (int j = 0; j < D; ++j) c[j] = j < dim ? coef[j] : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double xi = x[i], fi = gx[i] - xi;
        double add = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
            if (j < dim && c[j] != 0.0) add += c[j] * (X[(size_t)j * n + i] + beta * F[(size_t)j * n + i]);
        double v = xi + beta * fi - add;
        if (clamp && v < DBL_EPSILON) v = DBL_EPSILON;
        x[i] = v;
    }
}

template <int D>
cudaError_t run_mix(MixState &m, double *x, const double *gx, double beta, int iter, int clamp, cudaStream_t st) {
    const int slot = (iter - 1) % m.dim;
    k_pulay_hist<D><<<MIX_BLOCKS, MIX_THREADS, 0, st>>>(x, gx, m.X, m.F, m.xold, m.fold, m.n, m.dim, slot,
                                                        iter == 1, m.part);
    k_pulay_solve<<<1, 32, 0, st>>>(m.part, MIX_BLOCKS, m.dim, slot, iter > m.dim, m.FtF, m.coef);
    k_pulay_apply<D><<<MIX_BLOCKS, MIX_THREADS, 0, st>>>(x, gx, m.X, m.F, m.coef, m.n, m.dim, beta, clamp);
    return cudaGetLastError();
}

}  // namespace

void pwk_mix_free(void *p) {
    MixState *m = (MixState *)p;
    if (!m) return;
    if (m->mem) cudaFree(m->mem);
    delete m;
}

extern "C" int pw_mix_pulay(pw_ctx *c, double *x, const double *gx, int64_t n, double beta, int iter, int mixdim,
                            int clamp) {
    if (!c) return PW_ERR_ARG;
    if (!x || !gx || n <= 0 || iter < 1 || mixdim < 1 || mixdim > MIX_MAX || x == gx)
        return pwk_fail_msg(c, PW_ERR_ARG, "pw_mix_pulay: bad arguments (n > 0, iter >= 1, 1 <= mixdim <= 16, x != gx)");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail_msg(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    void **slot = pwk_mix_slot(c);
    MixState *m = (MixState *)*slot;
    if (!m || m->n != n || m->dim != mixdim) {
        if (iter != 1)
            return pwk_fail_msg(c, PW_ERR_STATE, "pw_mix_pulay: a new history (size or mixdim changed) must start at iter 1");
        if (m) {
            cudaStreamSynchronize(st);
            pwk_mix_free(m);
            *slot = nullptr;
        }
        m = new MixState();
        const size_t dn = (size_t)mixdim * n;
        const size_t doubles = 2 * dn + 2 * (size_t)n + (size_t)MIX_BLOCKS * 2 * mixdim + (size_t)mixdim * mixdim + mixdim;
        if (cudaMalloc(&m->mem, doubles * sizeof(double)) != cudaSuccess) {
            delete m;
            return pwk_fail_msg(c, PW_ERR_NOMEM, "pw_mix_pulay: no device memory for the history");
        }
        double *p = (double *)m->mem;
        m->X = p;
        m->F = p + dn;
        m->xold = p + 2 * dn;
        m->fold = m->xold + n;
        m->part = m->fold + n;
        m->FtF = m->part + (size_t)MIX_BLOCKS * 2 * mixdim;
        m->coef = m->FtF + (size_t)mixdim * mixdim;
        m->n = n;
        m->dim = mixdim;
        *slot = m;
    }
    if (iter == 1) {
        // a fresh history: empty slots read as zero columns of F
        if (cudaMemsetAsync(m->mem, 0, (2 * (size_t)mixdim * n) * sizeof(double), st) != cudaSuccess ||
            cudaMemsetAsync(m->FtF, 0, (size_t)mixdim * mixdim * sizeof(double), st) != cudaSuccess)
            return pwk_fail_msg(c, PW_ERR_CUDA, "pw_mix_pulay: cudaMemsetAsync failed");
    }
    cudaError_t e;
    if (mixdim <= 4)
        e = run_mix<4>(*m, x, gx, beta, iter, clamp, st);
    else if (mixdim <= 8)
        e = run_mix<8>(*m, x, gx, beta, iter, clamp, st);
    else
        e = run_mix<16>(*m, x, gx, beta, iter, clamp, st);
    if (e != cudaSuccess) return pwk_fail_msg(c, PW_ERR_CUDA, cudaGetErrorString(e));
    pwk_count_launches(c, 3);
    return PW_OK;
}
