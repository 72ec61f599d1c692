// Host-side launcher declarations shared by the kernel files and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "pw_common.cuh"

namespace pwk {

// Grow-only scratch slots of a context (pwk_scratch).  One list for every
// file so no two callers share a slot by accident; a slot is only reused by
// calls that never run at the same time as its other owner.
enum ScratchSlot {
    // update!: Poisson, XC, V_tot, reductions
    SL_UPD_A = 8, SL_UPD_RHOG, SL_UPD_VH, SL_UPD_VXC, SL_UPD_EPS, SL_UPD_VTOT, SL_UPD_RED,
    // update! with PBE: grad rho / h (3 x N), div h on the density sphere
    SL_UPD_GRAD, SL_UPD_DIVG,
    // band energies
    SL_BAND_W, SL_BAND_RED,
    // LOBPCG / generalized eigenproblem / ortho_sqrt
    SL_LOB_Q, SL_LOB_HQ, SL_LOB_TMP1, SL_LOB_TMP2, SL_LOB_SMALL, SL_LOB_EIGW, SL_LOB_EIGSTAT,
    // host drop-in staging of pw_lobpcg_host
    SL_HOST_C128, SL_HOST_C64,
    // forces
    SL_FRC_A, SL_FRC_B, SL_FRC_C,
    // adjoint of op_V_loc with respect to V (polarised blocks)
    SL_VJP,
    SL_COUNT
};
static_assert(SL_COUNT <= 32, "pw_ctx holds 32 scratch slots");

// Everything a pruned-FFT launch needs for one k-point and one precision.
struct FftLaunch {
    KPlan kp;
    FftDim dx, dy, dz;
    const void *twx, *twy, *twz;  // twiddle tables of the launch precision
    int Cg;                       // columns per CTA in the z passes
    int Jc;                       // y lines per x chunk in the plane passes
    int bpc = 1;                  // bands of one z-plane per CTA in the FP32 plane pass (1..3)
};

template <typename T> cudaError_t launch_zinv(const FftLaunch &, const void *psi, int64_t ld, int nb, void *A, cudaStream_t);
template <typename T>
cudaError_t launch_zfwd(const FftLaunch &, const void *A, const void *psi, void *Hpsi, int64_t ld, int nb, int flags,
                        cudaStream_t);
template <typename T> cudaError_t launch_plane_vloc(const FftLaunch &, const void *Vr, void *A, int nb, cudaStream_t);
// One projector column of betaNL (PsPotNL.jl:147-195 order): its atom,
// angular momentum l, m in [-l, l], radial index i (1-based), r_l and the
// normalisation of eval_proj_G.
struct ProjCol {
    int atom, l, m, i;
    double rc, pref;
};
cudaError_t launch_build_beta(const double *gk, int ngw, const ProjCol *cols, int ncol, const double *pos, double2 *beta,
                              cudaStream_t st);

template <typename T>
cudaError_t launch_multik(const FftLaunch &L, const MkK *ks, const int *band_k, int nk, int nbands, int max_nb,
                          int max_ncol, const void *Vr, void *A, int flags, const int *Drow, const int *Dcol,
                          const double *Dval, int nbeta, cudaStream_t st);
template <typename T>
cudaError_t launch_multik_persistent(const FftLaunch &L, const MkK *ks, const int *band_k, int nbands, int max_ncol,
                                     const void *Vr, void *A, int flags, const int *Drow, const int *Dcol,
                                     const double *Dval, int nbeta, unsigned *ctr, int *err, cudaStream_t st);
template <typename T>
cudaError_t launch_plane_rho(const FftLaunch &, const void *A, int nb, int G, int Bg, const double *w, void *rho_part,
                             cudaStream_t);
template <typename T> cudaError_t launch_rho_reduce(const void *part, int G, size_t N, double *rho, int acc, cudaStream_t);
template <typename T>
cudaError_t launch_opK(int Ngw, int nb, const double *Gk2, const void *psi, void *Hpsi, int64_t ld, int acc, cudaStream_t);
template <typename T>
cudaError_t launch_kprec(int Ngw, int nb, const double *Gk2, const void *in, void *out, int64_t ld, cudaStream_t);
template <typename T> cudaError_t launch_zero(void *p, int Ngw, int nb, int64_t ld, cudaStream_t);
template <typename T>
cudaError_t launch_polarize(int Ngw, int nb, const void *psi, const void *lam, int64_t ld, void *out, cudaStream_t);

// C (m x n, double2, ldc) (+)= A^H B with A (K x m), B (K x n) of element Cx<T>.
// ws: split-K workspace of at least gemm_tn_ws_bytes() bytes.
size_t gemm_tn_ws_bytes(int64_t K, int m, int n);
template <typename T>
// upper != 0: only C[i][j] with i <= j is formed and written (Hermitian
// products whose consumer reads the upper triangle); tiles strictly below
// the diagonal are skipped.
cudaError_t gemm_tn(int64_t K, int m, int n, const void *A, int64_t lda, const void *B, int64_t ldb, double2 *C,
                    int64_t ldc, int accumulate, void *ws, cudaStream_t, int upper = 0);
// C (M x n, Cx<T>, ldc) (+)= A (M x k, Cx<T>) * B (k x n, double2); tri: 1 = A
// lower triangular, 2 = B upper triangular and only C's upper triangle
// needed, 3 = A upper triangular (zero blocks skipped)
template <typename T>
cudaError_t gemm_nn(int64_t M, int n, int k, const void *A, int64_t lda, const double2 *B, int64_t ldb, void *C,
                    int64_t ldc, int accumulate, cudaStream_t, int tri = 0);
// P2[i][b] = sum_j D[i][j] P[j][b]  (CSR D; P, P2 are nbeta x nb, ld = nbeta)
cudaError_t apply_dcsr(int nbeta, int nb, const int *rowptr, const int *col, const double *val, const double2 *P,
                       double2 *P2, cudaStream_t);
// dtype conversions for the host drop-ins
cudaError_t convert_c128_to_c64(const double2 *in, float2 *out, size_t n, cudaStream_t);
cudaError_t convert_c64_to_c128(const float2 *in, double2 *out, size_t n, cudaStream_t);
cudaError_t convert_d_to_f(const double *in, float *out, size_t n, double scale, cudaStream_t);
cudaError_t scale_d(const double *in, double *out, size_t n, double scale, cudaStream_t);

}  // namespace pwk
