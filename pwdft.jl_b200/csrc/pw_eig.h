// FP64 small dense Hermitian eigensolver (see pw_eig.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace pwk {

// Bytes of device workspace hegv_lowest needs for order n, k eigenpairs.
size_t eig_work_bytes(int n, int k);

// Lowest k eigenpairs of T S = G S diag(lam) (G == nullptr: T S = S diag(lam)).
// T, G: n x n complex FP64 (column-major, device), read from their upper
// triangles and overwritten.  lam: device k doubles (ascending).  S: device
// n x k (column-major, ld n), S^H G S = I; S == nullptr: eigenvalues only.
// gemm_ws: unused (reserved).  d_status[0] != 0: a bounded grid barrier
// expired; d_status[1] = j > 0: G not positive definite at column j.
cudaError_t hegv_lowest(double2 *T, double2 *G, int n, int k, double *lam, double2 *S, void *work, size_t work_bytes,
                        void *gemm_ws, int *d_status, cudaStream_t st);

// Rinv = R^-1 for the Hermitian C = R^H R (C read from its upper triangle and
// overwritten), i.e. the inverse of cholesky(Hermitian(C)).U.  work: at least
// eig_work_bytes(n, 1) bytes.
cudaError_t chol_inverse_upper(double2 *C, int n, double2 *Rinv, void *work, int *d_status, cudaStream_t st);

}  // namespace pwk
