// Tensor-core (tcgen05) complex GEMM of the mixed-precision path; see pw_umma.cu.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pwk {

// A K-major split-BF16 operand: `rows` rows of Kp BF16 values per piece
// (hi, lo, and optionally a third piece lo2).  A product runs with three
// pieces (6 MMAs, ~2^-24) when both operands carry lo2, else with two
// (3 MMAs, ~2^-17).
struct UmmaOperand {
    __nv_bfloat16 *hi = nullptr;
    __nv_bfloat16 *lo = nullptr;
    __nv_bfloat16 *lo2 = nullptr;
    int64_t rows = 0;
    int Kp = 0;
    int rstride = 1;   // row r of a piece at r * rstride * Kp (2: the even rows of
                       // an A' operand, which are the B' rows of the same block)
};

int umma_kpad(int64_t K);                          // padded 2K (multiple of 64)
size_t umma_operand_bytes(int64_t rows, int64_t K);  // hi + lo bytes for `rows` rows (one piece: half)
// split-K count (splits > 0 overrides the automatic choice) and its
// workspace; a single split that does not accumulate writes the result
// directly (no finalize launch)
// (upper: the product is Hermitian and only tiles on or above the diagonal run)
int umma_splits(int64_t Mp, int Np, int Kp, int splits = 0, int upper = 0);
size_t umma_ws_bytes(int64_t Mp, int Np, int Kp, int splits = 0, int upper = 0);

// Operand builders (CT = float2 or double2 input element).
//   tn_a: A' (2m rows) from Z (K x m)          for C = Z^H W
//   tn_b: B' (n rows)  from W (K x n)
//   nn_a: A' (2M rows) from Z = A^H, A (M x k) for C = A U
template <typename CT> cudaError_t umma_prep_tn_a(const void *Z, int64_t ld, int64_t K, int m, UmmaOperand &, cudaStream_t);
template <typename CT> cudaError_t umma_prep_tn_b(const void *W, int64_t ld, int64_t K, int n, UmmaOperand &, cudaStream_t);
template <typename CT> cudaError_t umma_prep_nn_a(const void *A, int64_t lda, int64_t M, int k, UmmaOperand &, cudaStream_t);

// C (m x n complex of type CT, ldc) (+)= result; A.rows == 2m, B.rows == n.
// err: device int set non-zero if a bounded wait in the kernel expired.
template <typename CT>
// upper != 0: C is Hermitian and only C[i][j], i <= j, is formed and written.
// lolo != 0 (two-piece operands from the same block, C = Z^H Z): add the
// lo*lo product, whose omission biases the diagonal |z|^2 low.
cudaError_t umma_gemm(const UmmaOperand &A, const UmmaOperand &B, int m, int n, void *C, int64_t ldc, int accumulate,
                      float *ws, int *err, cudaStream_t, int upper = 0, int lolo = 0, int splits = 0);

}  // namespace pwk
