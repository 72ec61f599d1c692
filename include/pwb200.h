/*
 * pwb200.h -- C ABI of libpwb200.so, the B200 (sm_100a) implementation of
 * PWDFT.jl's Hamiltonian-application / density / eigensolver hot path.
 *
 * Every entry point returns an int status (PW_OK = 0); on failure the
 * message is available from pw_last_error(ctx).  No torch, Julia or C++
 * types cross this boundary: plain pointers, sizes and int flags only.
 *
 * Conventions shared with the reference (PWDFT.jl):
 *   - wavefunctions are column-major (Ngw x Nstates) complex arrays, the
 *     layout of Julia's Matrix{ComplexF64} (interleaved re, im);
 *   - grid linear index ip = i + N1*(j + N2*k), x fastest (PWGrid.jl:212);
 *   - G_to_R is the 1/N-normalised backward FFT, R_to_G the unnormalised
 *     forward FFT (wrappers_fft.jl:42-62);
 *   - op_* entry points ACCUMULATE into Hpsi when PW_ACCUMULATE is set
 *     (the reference's op_K!/op_V_loc!/op_V_Ps_nloc! semantics), and
 *     overwrite otherwise (op_H!, which zero-fills first, op_H.jl:53-63).
 *
 * Device entry points take device pointers and are ordered on the
 * context's stream (pw_set_stream); host entry points (suffix _host) take
 * host pointers to the reference's FP64 arrays and copy in and out.
 */
#ifndef PWB200_H
#define PWB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PWB200_ABI_VERSION 1

/* ---- status codes --------------------------------------------------- */
#define PW_OK               0
#define PW_ERR_ARG          1   /* invalid argument (size, index, pointer) */
#define PW_ERR_CUDA         2   /* a CUDA runtime call failed */
#define PW_ERR_NOMEM        3   /* device allocation failed */
#define PW_ERR_NOT_POSDEF   4   /* Cholesky of an overlap matrix failed */
#define PW_ERR_NAN          5   /* non-finite value in a reduction */
#define PW_ERR_STATE        6   /* call out of order (e.g. no V_loc set) */
#define PW_ERR_UNSUPPORTED  7   /* grid size with a prime factor > 5, ... */
#define PW_ERR_TIMEOUT      8   /* a bounded device-side wait gave up */

/* ---- element types of wavefunction buffers -------------------------- */
#define PW_C128  0   /* ComplexF64: the reference's type (FP64 path)   */
#define PW_C64   1   /* ComplexF32: mixed-precision path (FP32 FFTs)   */

/* ---- operator selection for pw_apply / pw_op_H_host ----------------- */
#define PW_OP_K        1u   /* op_K!        op_K.jl:44-75          */
#define PW_OP_VLOC     2u   /* op_V_loc!    op_V_loc.jl:108-167    */
#define PW_OP_VNL      4u   /* op_V_Ps_nloc! op_V_Ps_nloc.jl:39-78 */
#define PW_OP_H        7u   /* op_H!        op_H.jl:53-63          */
#define PW_ACCUMULATE  0x100u
#define PW_GRAPH       0x200u   /* pw_apply_multi: replay a captured CUDA graph */
#define PW_PERSISTENT  0x400u   /* pw_apply_multi: every stage in one cooperative launch */

typedef struct pw_ctx pw_ctx;

/* Basis description handed over once per Hamiltonian (PWGrid.gvecw). */
typedef struct pw_grid_desc {
    int32_t Ns[3];                  /* FFT grid (PWGrid.Ns)                     */
    int32_t Nkpt;                   /* number of k-points                        */
    int32_t Nspin;                  /* spin channels of V_loc (1 or 2)           */
    int32_t index_base;             /* 1: idx_gw2r is Julia 1-based, 0: 0-based  */
    double  CellVolume;             /* PWGrid.CellVolume (bohr^3)                */
    const int64_t *Ngw;             /* [Nkpt]            GVectorsW.Ngw           */
    const int64_t *const *idx_gw2r; /* [Nkpt][Ngw[k]]    GVectorsW.idx_gw2r      */
    const double *const *Gk2;       /* [Nkpt][Ngw[k]]    |G+k|^2 (op_K.jl:70)    */
} pw_grid_desc;

/* ---- library and context -------------------------------------------- */
int         pw_abi_version(void);

/* Replaces the FFTW plans and index maps carried by PWGrid
 * (PWGrid.jl:62-152): builds the pruned-FFT column tables on the host and
 * uploads them to `device`. */
int         pw_create(int device, const pw_grid_desc *desc, pw_ctx **out);
void        pw_destroy(pw_ctx *ctx);
const char *pw_last_error(const pw_ctx *ctx);
int         pw_set_stream(pw_ctx *ctx, void *cuda_stream);   /* cudaStream_t */
int         pw_synchronize(pw_ctx *ctx);
/* Number of kernels this context has launched so far (for launch
 * accounting in benchmarks; no counterpart in the reference). */
int64_t     pw_launch_count(const pw_ctx *ctx);
/* Synchronises the context's stream and reports PW_ERR_TIMEOUT if a bounded
 * device-side wait in one of its kernels gave up (no counterpart in the
 * reference, whose BLAS calls cannot time out). */
int         pw_check_device(pw_ctx *ctx);

/* Device buffers and copies for hosts that have no GPU array type of their
 * own (the Julia binding without CUDA.jl; no counterpart in the reference,
 * whose arrays all live on the host).  A buffer belongs to the context and
 * is freed by pw_device_free or pw_destroy; the copies are ordered on the
 * context stream and complete before the call returns. */
int pw_device_alloc(pw_ctx *ctx, uint64_t bytes, void **dptr);
int pw_device_free(pw_ctx *ctx, void *dptr);
int pw_copy_to_device(pw_ctx *ctx, void *dst, const void *src, uint64_t bytes);
int pw_copy_to_host(pw_ctx *ctx, void *dst, const void *src, uint64_t bytes);

/* Launch parameters of a context's kernels.  No counterpart in the
 * reference: there FFTW's planner and the BLAS pick their own blockings.
 * A zero field means "the built-in default"; pw_set_tuning replaces all
 * fields at once (read them with pw_get_tuning first to change one);
 * pw_get_tuning reports the band batch in effect (48 MiB by default). */
typedef struct pw_tuning {
    int64_t band_chunk_bytes; /* FFT intermediate of one band batch (default 48 MiB)             */
    int32_t plane_bands;      /* bands of one z-plane per CTA, FP32 plane pass: 1..3
                                 (default 3 on 75-point grids, else 1)                           */
    int32_t z_columns;        /* grid columns per CTA of the z passes, 1..256 (default: 64 for
                                 FP32, about 48 KB of shared memory for FP64)                    */
    int32_t gemm_splits;      /* split-K count of the tensor-core Gram and rotation, 0..64
                                 (0: enough CTAs to fill the GPU twice)                          */
    int32_t reserved[5];      /* must be zero                                                    */
} pw_tuning;
int pw_get_tuning(const pw_ctx *ctx, pw_tuning *t);
int pw_set_tuning(pw_ctx *ctx, const pw_tuning *t);

/* Autotuner of the launch parameters above for op_H (PW_OP_H) of k-point
 * ik on nb bands of dtype and, for PW_C64 with nb > 0, the Rayleigh-Ritz
 * Gram (3 nb x 3 nb over Ngw[ik]) and rotation (Ngw x 3nb -> nb).  Every
 * candidate is timed with CUDA events on the context stream on seeded
 * blocks the call allocates and frees, starting from the built-in defaults
 * (the context's current setting is not a candidate); the fastest set is
 * applied to the context and written to *chosen.  cache_path (NULL: the environment
 * variable PW_AUTOTUNE_CACHE, or no cache if unset) names a text file of
 * earlier choices keyed by GPU name, grid, Ngw, active columns and x
 * planes, nb, dtype and projector count: a hit applies the stored choice
 * without timing, a miss appends the new one.  ms (host, 4 doubles, may be
 * NULL) receives {op_H default, op_H tuned, Gram+rotation default,
 * Gram+rotation tuned} in milliseconds (negative when not timed, e.g. on a
 * cache hit).  No counterpart in the reference. */
int pw_autotune(pw_ctx *ctx, int ik, int nb, int dtype, const char *cache_path,
                pw_tuning *chosen, double *ms);

/* V_loc(r) = Ham.potentials.Total[:, ispin] (Hamiltonian.jl:542), host
 * FP64, N x nspin column-major.  Replaces the potential read by
 * op_V_loc.jl:127. */
int pw_set_vloc(pw_ctx *ctx, const double *V, int nspin);
int pw_set_vloc_device(pw_ctx *ctx, const double *V_dev, int nspin);

/* betaNL[ik] (PsPotNL.jl:39-69): host ComplexF64 Ngw x nbeta column-major. */
int pw_set_nonlocal(pw_ctx *ctx, int ik, const double *betaNL, int nbeta);
/* betaNL[ik] built on the device (PsPotNL.jl:16-77 for GTH: eval_proj_G,
 * PsPot_GTH.jl:338-391; Ylm_real, Ylm_real.jl:5-107; e^{-i(G+k).tau}) from
 * the G+k vectors of pw_set_gkvec and a host table of nbeta columns in the
 * reference's (atom, l, m, iprj) order: atom (0-based), l <= 3, m in
 * [-l, l], iproj (1-based radial index), rc = r_l of the atom's species,
 * pref = 4 pi^(5/4) sqrt(2^(l+1) r_l^(2l+3) / CellVolume); pos (host,
 * 3 x natoms, bohr).  Replaces pw_set_nonlocal's host array, e.g. after the
 * atoms moved. */
int pw_build_nonlocal(pw_ctx *ctx, int ik, int nbeta, const int32_t *atom,
                      const int32_t *l, const int32_t *m, const int32_t *iproj,
                      const double *rc, const double *pref, int natoms,
                      const double *pos);
/* The (ibeta, jbeta, h_ij) pairs visited by op_V_Ps_nloc.jl:59-76
 * (0-based ibeta/jbeta; duplicates add). */
int pw_set_nonlocal_coef(pw_ctx *ctx, int nnz, const int32_t *ibeta,
                         const int32_t *jbeta, const double *hij);

/* ---- device entry points (device pointers, context stream) ---------- */

/* Hpsi (+)= H psi restricted to `ops` for k-point ik (0-based), spin
 * ispin (0-based); psi/Hpsi are Ngw[ik] x nb with leading dimension ld.
 * dtype PW_C128 computes in FP64, PW_C64 in FP32 (mixed precision).
 * Replaces op_H!/op_K!/op_V_loc!/op_V_Ps_nloc! (op_H.jl:53-63). */
int pw_apply(pw_ctx *ctx, int ik, int ispin, int dtype, const void *psi,
             void *Hpsi, int64_t ld, int nb, unsigned ops);

/* The BlochWavefunc form op_H!(Ham, psiks, Hpsiks) (op_H.jl:4-35,
 * op_K.jl:17-29, op_V_loc.jl:17-28, op_V_Ps_nloc.jl:22-37) for spin
 * ispin: Hpsi[i] (+)= H(k = iks[i]) psi[i] for nk k-points in one launch
 * per stage (their Ngw differ).  psi, Hpsi: host arrays of nk device
 * pointers (Ngw x nb[i], leading dimension ld[i]).  ops must contain
 * PW_OP_VLOC (op_K and op_V_Ps_nloc optional, PW_ACCUMULATE as pw_apply);
 * cube grids of 27, 75 or 120 points, at most 65535 bands and 2048
 * projectors.  With PW_GRAPH the launches are captured in a CUDA graph and
 * a later call with the same k-points, blocks, flags and buffers replays
 * it.  With PW_PERSISTENT all stages run in one cooperative launch whose
 * CTAs loop over the work of each stage, separated by bounded grid
 * barriers (it falls back to the per-stage launches when one CTA per SM
 * does not fit); the per-stage launches are the default because they
 * measured faster (the fused kernel holds the registers of its largest
 * stage throughout). */
int pw_apply_multi(pw_ctx *ctx, int nk, const int *iks, int ispin, int dtype,
                   void *const *psi, void *const *Hpsi, const int64_t *ld,
                   const int *nb, unsigned ops);

/* out = in / (1 + |G+k|^2)  (Kprec.jl:30-44; in == out allowed). */
int pw_kprec(pw_ctx *ctx, int ik, int dtype, const void *in, void *out,
             int64_t ld, int nb);

/* rhoe[ip] (+)= sum_b w[b] |(N/sqrt(Omega)) G_to_R(psi_b)|^2
 * (calc_rhoe.jl:51-78); w (host, nb) = wk[ik]*Focc[b, ikspin]; rhoe is a
 * device FP64 array of N points (one spin channel).  accumulate = 0
 * overwrites. */
int pw_calc_rhoe(pw_ctx *ctx, int ik, int dtype, const void *psi, int64_t ld,
                 int nb, const double *w, double *rhoe, int accumulate);

/* Adjoint of op_V_loc! (op_V_loc.jl:33-92) with respect to the potential:
 *   dV[r] (+)= sum_b w[b] N Re( conj(G_to_R(lam_b))[r] G_to_R(psi_b)[r] ),
 * the gradient of L = sum_b w_b Re<lam_b| V_loc psi_b> with respect to the
 * V_loc(r) of pw_set_vloc.  lam == psi (or NULL) gives dE/dV_loc(r) of the
 * band energy E = sum_b w_b <psi_b|H|psi_b> (w = wk * Focc): the density of
 * calc_rhoe.jl:51-78 times dVol = Omega/N, the quantity that
 * calc_forces_Ps_loc.jl:13-72 contracts with dV_ps/dtau and, at self
 * consistency, the derivative of the total energy with respect to an
 * external potential.  psi, lam: device Ngw x nb (ld) of dtype; w: host nb;
 * dV: device FP64, N points; accumulate = 0 overwrites. */
int pw_vloc_vjp(pw_ctx *ctx, int ik, int dtype, const void *psi, const void *lam,
                int64_t ld, int nb, const double *w, double *dV, int accumulate);

/* Rayleigh-Ritz contractions (diag_LOBPCG.jl:85,144,152-153,183-184):
 * C (m x n, device ComplexF64, ldc) (+)= A^H B, A is K x m, B is K x n,
 * both of element type dtype. */
int pw_gram(pw_ctx *ctx, int dtype, int64_t K, int m, int n, const void *A,
            int64_t lda, const void *B, int64_t ldb, double *C, int64_t ldc,
            int accumulate);
/* C (M x n, dtype, ldc) (+)= A (M x k, dtype, lda) * U (k x n, device
 * ComplexF64, ldu)  (diag_LOBPCG.jl:188-194). */
int pw_rotate(pw_ctx *ctx, int dtype, int64_t M, int n, int k, const void *A,
              int64_t lda, const double *U, int64_t ldu, void *C, int64_t ldc,
              int accumulate);

/* Allocation-free variant of pw_apply for the local-potential round trip
 * (ops = PW_OP_VLOC, optionally | PW_OP_K | PW_ACCUMULATE).  It has no
 * counterpart in the reference.  It is for callers that cannot allocate
 * device memory on this path: a host that hands the whole GPU to its own
 * pooling allocator, or a solver loop that must not stall on the implicit
 * device synchronisation of cudaMalloc/cudaFree.  pw_apply may grow its
 * intermediate buffer on first use or when nb grows; this call never does.
 * Its intermediate is one file-scope device array of
 * pw_noalloc_scratch_bytes() (32 MiB).  pw_create looks up the array's
 * device address on its device, which loads it there: from the first
 * pw_create on a GPU the 32 MiB stay reserved until the process exits (so
 * create the context before a pooling allocator takes the GPU's memory),
 * and this call itself reserves nothing.  Bands are processed in batches
 * that fit, and a grid whose single band needs more returns
 * PW_ERR_UNSUPPORTED.  All calls share the array, so calls whose work
 * overlaps on the GPU (other streams, other contexts) race. */
int      pw_apply_vloc_noalloc(pw_ctx *ctx, int ik, int ispin, int dtype,
                               const void *psi, void *Hpsi, int64_t ld,
                               int nb, unsigned ops);
uint64_t pw_noalloc_scratch_bytes(void);

/* Lowest k eigenpairs of the Hermitian-definite pencil (T, G) of order n,
 * FP64 on the device: T S = G S diag(lam), S^H G S = I (G == NULL: standard
 * problem T S = S diag(lam)).  T and G are read from their upper triangles
 * (Julia's Hermitian(A)) and overwritten; lam: device k doubles ascending;
 * S: device n x k ComplexF64 or NULL for eigenvalues only.  Replaces
 * eigen(T, G) / eigvals(XHX) / eigen(S) of diag_LOBPCG.jl:86,185,216.
 * PW_ERR_NOT_POSDEF when G is not positive definite. */
int pw_eigh(pw_ctx *ctx, int n, int k, double *T, double *G, double *lam,
            double *S);

/* diag_LOBPCG!(Ham, X; tol, NiterMax, Nstates_conv) for k-point ik
 * (diag_LOBPCG.jl:51-225): X (device, Ngw x nb, ld) is overwritten with the
 * Ritz vectors, evals (host, nb) with the Ritz values; converged when
 * nconv (or nb if nconv <= 0) eigenvalues moved by less than tol between
 * iterations.  dtype PW_C64 runs the blocks in FP32 with split-BF16x3
 * tensor-core contractions and FP64 small matrices; PW_C128 is all FP64.
 * niter (host, may be NULL) receives the iteration count. */
int pw_lobpcg(pw_ctx *ctx, int ik, int ispin, int dtype, void *X, int64_t ld,
              int nb, double tol, int nitermax, int nconv, double *evals,
              int *niter);

/* diag_davidson_qe!(Ham, evc; EBANDS_THR = tol, NiterMax = nitermax) for
 * k-point ik (diag_davidson_qe_v2.jl:38-216): the QE-style block Davidson
 * with Nvecx = 2 nb and restart, S = identity (norm-conserving).  X (device,
 * Ngw x nb, ld) is overwritten with the Ritz vectors evc, evals (host, nb)
 * with the Ritz values; a root is converged when its Ritz value moved by
 * less than tol in an iteration.  Needs 2 nb <= Ngw.  dtype as pw_lobpcg;
 * niter (host, may be NULL) receives the iteration count (+1000 when the
 * mixed-precision reduced overlap lost definiteness and the iteration
 * stopped on the previous step's Ritz vectors). */
int pw_davidson(pw_ctx *ctx, int ik, int ispin, int dtype, void *X, int64_t ld,
                int nb, double tol, int nitermax, double *evals, int *niter);

/* chebyfilt(Ham, X, degree, lb, ub) for k-point ik (CheFSI.jl:34-64): the
 * scaled Chebyshev filter of the given degree (>= 1) over [lb, ub]
 * (ub > lb), Y = p(H) X with the three-term recurrence of the reference
 * (sigma1 = e / (lb - ub) fixed, sigma_{i+1} = 1 / (2 / sigma1 - sigma_i)).
 * X and Y: distinct device blocks Ngw x nb (ld) of dtype; X is left
 * unchanged.  degree op_H applications plus one fused combination kernel
 * per step. */
int pw_chebyfilt(pw_ctx *ctx, int ik, int ispin, int dtype, const void *X,
                 void *Y, int64_t ld, int nb, int degree, double lb,
                 double ub);

/* get_ub_lb_lanczos(Ham, nlancz) for k-point ik (CheFSI.jl:67-125, with
 * norm_matrix_induced of :127-137): nlancz (even, <= Ngw) Lanczos steps
 * from the start vector v0 (device, Ngw ComplexF64; the reference draws it
 * with randn) with one step of full reorthogonalisation, in FP64.
 * lb = the (nlancz/2)-th smallest eigenvalue of the Lanczos matrix T,
 * ub = ||T 1/sqrt(nlancz)|| + ||f|| (host doubles).  T's eigenvalues come
 * from the Hermitian device solver on its upper triangle, which equals the
 * reference's general eigvals(T) to rounding.  PW_ERR_NAN on a Lanczos
 * breakdown (zero residual). */
int pw_lanczos_bounds(pw_ctx *ctx, int ik, int ispin, int nlancz,
                      const double *v0, double *lb, double *ub);

/* diag_LOBPCG! over many k-points at once (diag_LOBPCG.jl:1-28 with the
 * per-k-point steps of :51-225, the FP64 path's order) for small blocks:
 * X[i] (device, Ngw[iks[i]] x nb, ld[i]) overwritten with the Ritz vectors,
 * evals (host, nb x nk, column i for k-point iks[i]).  Every step is one
 * launch for all k-points; a k-point stops where its own test
 * |lambda - lambda_old| < tol holds for nconv (nb if <= 0) values.
 * Needs 3 nb <= 48.  niter: iterations of the slowest k-point. */
int pw_lobpcg_multi(pw_ctx *ctx, int nk, const int *iks, int ispin, int dtype,
                    void *const *X, const int64_t *ld, int nb, double tol,
                    int nitermax, int nconv, double *evals, int *niter);

/* ---- update! and energies on the device ----------------------------- */

/* The density G-sphere (PWGrid.gvec: idx_g2r, G2, sorted by G2 so that
 * G = 0 comes first, PWGrid.jl:199-242), needed by pw_poisson/pw_update. */
int pw_set_density_sphere(pw_ctx *ctx, int64_t Ng, const int64_t *idx_g2r,
                          const double *G2, int index_base);
/* Exchange-correlation of pw_update: the reference's internal functionals
 * (Hamiltonian.jl:270-277, use_xc_internal = true): PW_XC_VWN (default;
 * LDA_VWN_internal.jl) or PW_XC_PBE (GGA_PBE_internal.jl:29-145, gradients
 * by PWGrid.jl:351-398 op_nabla / op_nabla_dot on the density sphere).
 * G (host, 3 x Ng, the sphere of pw_set_density_sphere in its order) is
 * required for PBE and ignored for VWN. */
#define PW_XC_VWN 0
#define PW_XC_PBE 1
int pw_set_xc(pw_ctx *ctx, int xc, const double *G);
/* RhoeSymmetrizer (RhoeSymmetrizer.jl:14-110) for symmetrize_rhoe!: the
 * orbits of the density sphere under the crystal's rotations, each given
 * as nsym entries (host): isg (nshell x nsym, 0-based sphere index of
 * inv_s g0 for each operation, g0 the orbit's first member) and phase
 * (nshell x nsym x 2: cos, sin of G_isg . ft_cartesian; 1, 0 for
 * symmorphic operations), in the reference's operation order. */
int pw_set_symmetry(pw_ctx *ctx, int nshell, int nsym, const int32_t *isg,
                    const double *phase);
/* symmetrize_rhoe! (RhoeSymmetrizer.jl:114-236), one spin channel, in
 * place on the device density rhoe (N): each orbit's rho(G) averaged with
 * the fractional-translation phases; grid components outside the density
 * sphere are kept. */
int pw_symmetrize_rhoe(pw_ctx *ctx, double *rhoe);

/* mix_pulay! (mix_pulay.jl:1-41) on device vectors, the history kept in the
 * context: x (device FP64, n) is the input density of SCF iteration iter
 * (1-based; iter == 1 starts a new history), gx (device, n, distinct) the
 * output density.  x is overwritten with x + beta f before iteration
 * mixdim + 1 and with x + beta f - (X + beta F) inv(F'F) F'f from then on
 * (f = gx - x; X, F the last mixdim differences), then clamped to >= eps()
 * when clamp != 0 (KS_solve_SCF.jl:277-281).  mixdim <= 16; a singular F'F
 * mixes simply for that iteration.  No host synchronisation. */
int pw_mix_pulay(pw_ctx *ctx, double *x, const double *gx, int64_t n, double beta,
                 int iter, int mixdim, int clamp);

/* Poisson_solve! (Poisson_solve.jl:22-40): V_H(r) from rho(r), device FP64
 * arrays of N points. */
int pw_poisson(pw_ctx *ctx, const double *rho, double *VH);
/* update! (Hamiltonian.jl:510-545, VWN or PBE per pw_set_xc, Nspin = 1) + the sums of
 * calc_E_local (calc_energies.jl:245-333): V_tot = V_ps + V_H + V_xc becomes
 * the context's V_loc; VH / Vxc (device N, may be NULL) receive V_H and
 * V_xc; E3 (host) = {sum V_H rho, sum V_ps rho, sum eps_xc rho} (multiply by
 * dVol, and E_Hartree by 1/2). */
int pw_update(pw_ctx *ctx, const double *rho, const double *Vps, double *VH,
              double *Vxc, double *E3);
/* calc_E_kin + calc_E_Ps_nloc (calc_energies.jl:342-375, 7-58) of one
 * k-point: E2 (host) = {0.5 sum_b w_b sum_g |psi|^2 |G+k|^2,
 * sum_b w_b sum_ij h_ij conj(B_i) B_j} with w (host, nb) = wk * Focc. */
int pw_band_energies(pw_ctx *ctx, int ik, int dtype, const void *psi,
                     int64_t ld, int nb, const double *w, double *E2);

/* ---- ionic forces --------------------------------------------------- */

/* Tables of calc_forces_Ps_loc! (calc_forces_Ps_loc.jl:20-57), once per
 * cell: G (host, 3 x Ng, the density sphere of pw_set_density_sphere in its
 * order) and VlocG (host, Ng x nspecies) = eval_Vloc_G of each species on
 * those G (without the 1/CellVolume factor, which cancels). */
int pw_set_force_tables(pw_ctx *ctx, int nspecies, const double *VlocG, const double *G);

/* calc_forces_Ps_loc! (calc_forces_Ps_loc.jl:13-71): F (host, 3 x natoms)
 * from rho (device, N) and the atoms' positions (host, 3 x natoms, bohr)
 * and species (host, 0-based). */
int pw_forces_local(pw_ctx *ctx, const double *rho, int natoms, const double *pos,
                    const int32_t *species, double *F);

/* The (G+k) vectors of k-point ik (host, 3 x Ngw in the idx_gw2r order),
 * used by calc_dbetaNL (calc_forces_Ps_nloc.jl:347-391). */
int pw_set_gkvec(pw_ctx *ctx, int ik, const double *gk);

/* Atom of each projector (host, NbetaNL, 0-based, nondecreasing as in
 * PsPotNL.jl:147-195). */
int pw_set_nonlocal_atoms(pw_ctx *ctx, int natoms, const int32_t *atom_of_beta);

/* calc_forces_Ps_nloc! for GTH (calc_forces_Ps_nloc.jl:291-411) of one
 * k-point: F (host, 3 x natoms) = sum_s 2 w_s Re(h_ij conj(B_i) dB_j) over
 * each atom's (ibeta, jbeta, h_ij), B = betaNL' psi, dB = dbetaNL' psi;
 * psi device Ngw x nb (ld), w (host, nb) = wk * Focc.  Overwrites F. */
int pw_forces_nonlocal(pw_ctx *ctx, int ik, int dtype, const void *psi, int64_t ld,
                       int nb, const double *w, double *F);

/* ortho_sqrt!(psi) (ortho_sqrt.jl:1-11): psi := psi * inv(sqrt(psi'psi)),
 * psi device Ngw x nb (ld), in place. */
int pw_ortho_sqrt(pw_ctx *ctx, int dtype, void *psi, int64_t ld, int64_t ngw,
                  int nb);

/* Rinv = inv(cholesky(Hermitian(C)).U): the upper-triangular factor that
 * diag_LOBPCG.jl:144-147,170-174,195-199 divides W and P by (W / R).  C (device,
 * n x n ComplexF64, upper triangle read) is overwritten; Rinv (device, n x n
 * column-major).  PW_ERR_NOT_POSDEF when C is not positive definite. */
int pw_chol_rinv(pw_ctx *ctx, int n, double *C, double *Rinv);

/* ortho_cholesky!(Ham, psi) (ortho_sqrt.jl:80-89): O = psi'psi = U^H U,
 * psi := psi / U, psi device Ngw x nb (ld), in place. */
int pw_ortho_cholesky(pw_ctx *ctx, int dtype, void *psi, int64_t ld, int64_t ngw, int nb);

/* calc_grad(Ham, psi) (calc_grad.jl:1-57) for k-point ik, spin ispin:
 * grad = wk f_i (H psi_i - sum_j psi_j <psi_j|H psi_i>), plus
 * psi (Hred F - F Hred)/2 when Focc (host, nb) is not all 2 or all 1.
 * psi and grad device Ngw x nb (ld), distinct. */
int pw_calc_grad(pw_ctx *ctx, int ik, int ispin, int dtype, const void *psi, void *grad,
                 int64_t ld, int nb, const double *Focc, double wk);

/* ---- host drop-ins (the reference's Julia arrays) ------------------- */

/* op_H!(Ham, psi, Hpsi) and friends on host ComplexF64 arrays; compute
 * precision chosen by dtype (PW_C128 = reference FP64, PW_C64 = mixed). */
int pw_op_H_host(pw_ctx *ctx, int ik, int ispin, const double *psi,
                 double *Hpsi, int64_t ld, int nb, unsigned ops, int dtype);
/* diag_LOBPCG!(Ham, X) for k-point ik on the reference's host array X
 * (Ngw x nb ComplexF64, ld), copied in and out around pw_lobpcg. */
int pw_lobpcg_host(pw_ctx *ctx, int ik, int ispin, int dtype, double *X,
                   int64_t ld, int nb, double tol, int nitermax, int nconv,
                   double *evals, int *niter);
/* diag_davidson_qe!(Ham, evc) for k-point ik on the reference's host array
 * evc (Ngw x nb ComplexF64, ld), copied in and out around pw_davidson. */
int pw_davidson_host(pw_ctx *ctx, int ik, int ispin, int dtype, double *X,
                     int64_t ld, int nb, double tol, int nitermax,
                     double *evals, int *niter);
/* calc_rhoe! inner loop for one k-point on host arrays; rhoe is host FP64
 * (N), accumulated when accumulate != 0. */
int pw_calc_rhoe_host(pw_ctx *ctx, int ik, const double *psi, int64_t ld,
                      int nb, const double *w, double *rhoe, int accumulate,
                      int dtype);

/* ---- host-side basis construction (no device) ----------------------- */

/* good_fft_order (fft_support.jl:48-72). */
int pw_good_fft_order(int n);
/* Number of G with 0.5|G|^2 <= ecutrho (PWGrid.jl:169-189); recvecs is
 * the 3x3 RecVecs matrix in Julia column-major order. */
int pw_gvec_count(const int32_t *Ns, const double *recvecs, double ecutrho,
                  int64_t *Ng);
/* init_gvec (PWGrid.jl:199-242): G (3 x Ng), G2, idx_g2r (0-based),
 * sorted by a stable sort on G2, bit-identical to the reference. */
int pw_gvec_build(const int32_t *Ns, const double *recvecs, double ecutrho,
                  int64_t Ng, double *G, double *G2, int64_t *idx_g2r);
/* init_gvecw for one k-point (PWGrid.jl:306-316): returns Ngw and fills
 * idx_gw2g / idx_gw2r (0-based) and Gk2 (capacity Ng each). */
int pw_gvecw_build(int64_t Ng, const double *G, const int64_t *idx_g2r,
                   const double *kpt, double ecutwfc, int64_t *Ngw,
                   int64_t *idx_gw2g, int64_t *idx_gw2r, double *Gk2);

#ifdef __cplusplus
}
#endif
#endif /* PWB200_H */
