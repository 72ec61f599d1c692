// Complex GEMMs on CUDA cores for the FP64 path (and the reference for the
// tensor-core kernels):
//   gemm_tn  C = A^H B      projections betaNL' psi (PsPotNL.jl:252) and the
//                           Rayleigh-Ritz Gram matrices X'HX, Q'HQ, Q'Q
//                           (diag_LOBPCG.jl:85,152-153,183-184); long K =
//                           Ngw is split across CTAs (deterministic two-pass
//                           reduction in FP64).
//   gemm_nn  C (+)= A B     betaNL * (D * P) (op_V_Ps_nloc.jl:59-76) and the
//                           subspace rotations Q*U, HQ*U (diag_LOBPCG.jl:188-194)
#include "pw_launch.h"

namespace pwk {

namespace {

constexpr int TN_BM = 32, TN_BN = 32, TN_BK = 32;

template <typename T>
__global__ void __launch_bounds__(256)
k_gemm_tn(int64_t K, int m, int n, const Cx<T> *__restrict__ A, int64_t lda, const Cx<T> *__restrict__ B, int64_t ldb,
          double2 *__restrict__ W, int64_t kchunk, int upper) {
    __shared__ Cx<T> As[TN_BK][TN_BM + 1];
    __shared__ Cx<T> Bs[TN_BK][TN_BN + 1];
    const int m0 = blockIdx.x * TN_BM, n0 = blockIdx.y * TN_BN;
    if (upper && m0 > n0 + TN_BN - 1) return;  // tile strictly below the diagonal
    const int64_t kbeg = (int64_t)blockIdx.z * kchunk;
    const int64_t kend = min(K, kbeg + kchunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    Cx<T> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j] = cmake((T)0, (T)0);
    for (int64_t k0 = kbeg; k0 < kend; k0 += TN_BK) {
        for (int e = threadIdx.x; e < TN_BK * TN_BM; e += 256) {
            const int kk = e % TN_BK, mm = e / TN_BK;
            const int64_t k = k0 + kk;
            As[kk][mm] = (k < kend && m0 + mm < m) ? A[(size_t)(m0 + mm) * lda + k] : cmake((T)0, (T)0);
            Bs[kk][mm] = (k < kend && n0 + mm < n) ? B[(size_t)(n0 + mm) * ldb + k] : cmake((T)0, (T)0);
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < TN_BK; ++kk) {
            Cx<T> a0 = As[kk][tx], a1 = As[kk][tx + 16];
            Cx<T> b0 = Bs[kk][ty], b1 = Bs[kk][ty + 16];
            acc[0][0] = cadd(acc[0][0], cmulc(a0, b0));
            acc[0][1] = cadd(acc[0][1], cmulc(a0, b1));
            acc[1][0] = cadd(acc[1][0], cmulc(a1, b0));
            acc[1][1] = cadd(acc[1][1], cmulc(a1, b1));
        }
        __syncthreads();
    }
    double2 *Wz = W + (size_t)blockIdx.z * m * n;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int mm = m0 + tx + 16 * i, nn = n0 + ty + 16 * j;
            if (mm < m && nn < n) Wz[(size_t)nn * m + mm] = make_double2((double)acc[i][j].x, (double)acc[i][j].y);
        }
}

__global__ void k_splitk_reduce(const double2 *__restrict__ W, int S, int m, int n, double2 *__restrict__ C, int64_t ldc,
                                int accumulate, int upper) {
    const size_t total = (size_t)m * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int nn = (int)(t / m), mm = (int)(t - (size_t)nn * m);
        if (upper && mm > nn) continue;
        double2 s = accumulate ? C[(size_t)nn * ldc + mm] : make_double2(0.0, 0.0);
        for (int z = 0; z < S; ++z) {
            const double2 v = W[(size_t)z * total + t];
            s.x += v.x;
            s.y += v.y;
        }
        C[(size_t)nn * ldc + mm] = s;
    }
}

constexpr int NN_BM = 64, NN_BN = 32, NN_BK = 16;

// tri: triangular structure the caller guarantees (the k-loop skips the
// zero blocks, whole tiles are skipped where no needed output lies):
//   1  A lower triangular (A[g][l] = 0 for l > g)
//   2  B upper triangular (B[l][j] = 0 for l > j) and only C[g][j], g <= j,
//      needed (tiles entirely below the diagonal are not formed)
//   3  A upper triangular (A[g][l] = 0 for l < g)
template <typename T>
__global__ void __launch_bounds__(256)
k_gemm_nn(int64_t M, int n, int k, const Cx<T> *__restrict__ A, int64_t lda, const double2 *__restrict__ B, int64_t ldb,
          Cx<T> *__restrict__ C, int64_t ldc, int accumulate, int tri) {
    __shared__ Cx<T> As[NN_BK][NN_BM];
    __shared__ Cx<T> Bs[NN_BK][NN_BN];
    const int64_t g0 = (int64_t)blockIdx.x * NN_BM;
    const int n0 = blockIdx.y * NN_BN;
    if (tri == 2 && g0 > n0 + NN_BN - 1) return;   // the whole CTA: before any barrier
    int jbeg = 0, jend = k;
    if (tri == 1) jend = (int)min((int64_t)k, g0 + NN_BM);
    if (tri == 2) jend = min(k, n0 + NN_BN);
    if (tri == 3) jbeg = (int)min((int64_t)k, (g0 / NN_BK) * NN_BK);
    const int tg = threadIdx.x & 63, tn = threadIdx.x >> 6;  // 64 rows x 4 column groups of 8
    Cx<T> acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = cmake((T)0, (T)0);
    for (int j0 = jbeg; j0 < jend; j0 += NN_BK) {
        for (int e = threadIdx.x; e < NN_BK * NN_BM; e += 256) {
            const int gg = e % NN_BM, jj = e / NN_BM;
            As[jj][gg] = (g0 + gg < M && j0 + jj < k) ? A[(size_t)(j0 + jj) * lda + g0 + gg] : cmake((T)0, (T)0);
        }
        for (int e = threadIdx.x; e < NN_BK * NN_BN; e += 256) {
            const int jj = e % NN_BK, nn = e / NN_BK;
            double2 v = (j0 + jj < k && n0 + nn < n) ? B[(size_t)(n0 + nn) * ldb + j0 + jj] : make_double2(0.0, 0.0);
            Bs[jj][nn] = cmake((T)v.x, (T)v.y);
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < NN_BK; ++jj) {
            const Cx<T> a = As[jj][tg];
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[q] = cadd(acc[q], cmul(a, Bs[jj][tn * 8 + q]));
        }
        __syncthreads();
    }
    const int64_t g = g0 + tg;
    if (g < M) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int nn = n0 + tn * 8 + q;
            if (nn < n) {
                Cx<T> *p = C + (size_t)nn * ldc + g;
                *p = accumulate ? cadd(*p, acc[q]) : acc[q];
            }
        }
    }
}

__global__ void k_dcsr(int nbeta, int nb, const int *__restrict__ rowptr, const int *__restrict__ col,
                       const double *__restrict__ val, const double2 *__restrict__ P, double2 *__restrict__ P2) {
    const size_t total = (size_t)nbeta * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / nbeta), i = (int)(t - (size_t)b * nbeta);
        double2 s = make_double2(0.0, 0.0);
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const double2 p = P[(size_t)b * nbeta + col[e]];
            s.x += val[e] * p.x;
            s.y += val[e] * p.y;
        }
        P2[t] = s;
    }
}

__global__ void k_c128_to_c64(const double2 *in, float2 *out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}
__global__ void k_c64_to_c128(const float2 *in, double2 *out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_double2((double)in[i].x, (double)in[i].y);
}
__global__ void k_d_to_f(const double *in, float *out, size_t n, double s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)(in[i] * s);
}
__global__ void k_scale_d(const double *in, double *out, size_t n, double s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[i] * s;
}

int blocks_for(size_t total) {
    size_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return b < 1 ? 1 : (int)b;
}

int splitk_count(int64_t K, int m, int n) {
    const int tiles = ((m + TN_BM - 1) / TN_BM) * ((n + TN_BN - 1) / TN_BN);
    int64_t S = (600 + tiles - 1) / tiles;
    const int64_t Smax = (K + 255) / 256;
    if (S > Smax) S = Smax;
    if (S < 1) S = 1;
    return (int)S;
}

}  // namespace

size_t gemm_tn_ws_bytes(int64_t K, int m, int n) {
    return (size_t)splitk_count(K, m, n) * m * n * sizeof(double2);
}

template <typename T>
cudaError_t gemm_tn(int64_t K, int m, int n, const void *A, int64_t lda, const void *B, int64_t ldb, double2 *C,
                    int64_t ldc, int accumulate, void *ws, cudaStream_t st, int upper) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    const int S = splitk_count(K, m, n);
    int64_t kchunk = (K + S - 1) / S;
    kchunk = ((kchunk + TN_BK - 1) / TN_BK) * TN_BK;
    dim3 grid((m + TN_BM - 1) / TN_BM, (n + TN_BN - 1) / TN_BN, S);
    k_gemm_tn<T><<<grid, 256, 0, st>>>(K, m, n, (const Cx<T> *)A, lda, (const Cx<T> *)B, ldb, (double2 *)ws, kchunk, upper);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_splitk_reduce<<<blocks_for((size_t)m * n), 256, 0, st>>>((const double2 *)ws, S, m, n, C, ldc, accumulate, upper);
    return cudaGetLastError();
}

template <typename T>
cudaError_t gemm_nn(int64_t M, int n, int k, const void *A, int64_t lda, const double2 *B, int64_t ldb, void *C,
                    int64_t ldc, int accumulate, cudaStream_t st, int tri) {
    if (M <= 0 || n <= 0) return cudaSuccess;
    dim3 grid((unsigned)((M + NN_BM - 1) / NN_BM), (n + NN_BN - 1) / NN_BN);
    k_gemm_nn<T><<<grid, 256, 0, st>>>(M, n, k, (const Cx<T> *)A, lda, B, ldb, (Cx<T> *)C, ldc, accumulate, tri);
    return cudaGetLastError();
}

template cudaError_t gemm_tn<float>(int64_t, int, int, const void *, int64_t, const void *, int64_t, double2 *, int64_t,
                                    int, void *, cudaStream_t, int);
template cudaError_t gemm_tn<double>(int64_t, int, int, const void *, int64_t, const void *, int64_t, double2 *, int64_t,
                                     int, void *, cudaStream_t, int);
template cudaError_t gemm_nn<float>(int64_t, int, int, const void *, int64_t, const double2 *, int64_t, void *, int64_t,
                                    int, cudaStream_t, int);
template cudaError_t gemm_nn<double>(int64_t, int, int, const void *, int64_t, const double2 *, int64_t, void *, int64_t,
                                     int, cudaStream_t, int);

cudaError_t apply_dcsr(int nbeta, int nb, const int *rowptr, const int *col, const double *val, const double2 *P,
                       double2 *P2, cudaStream_t st) {
    k_dcsr<<<blocks_for((size_t)nbeta * nb), 256, 0, st>>>(nbeta, nb, rowptr, col, val, P, P2);
    return cudaGetLastError();
}
cudaError_t convert_c128_to_c64(const double2 *in, float2 *out, size_t n, cudaStream_t st) {
    k_c128_to_c64<<<blocks_for(n), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t convert_c64_to_c128(const float2 *in, double2 *out, size_t n, cudaStream_t st) {
    k_c64_to_c128<<<blocks_for(n), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t convert_d_to_f(const double *in, float *out, size_t n, double scale, cudaStream_t st) {
    k_d_to_f<<<blocks_for(n), 256, 0, st>>>(in, out, n, scale);
    return cudaGetLastError();
}
cudaError_t scale_d(const double *in, double *out, size_t n, double scale, cudaStream_t st) {
    k_scale_d<<<blocks_for(n), 256, 0, st>>>(in, out, n, scale);
    return cudaGetLastError();
}

}  // namespace pwk
