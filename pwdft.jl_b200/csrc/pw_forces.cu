// Ionic forces on the device: the local and nonlocal pseudopotential terms.
//
//   local   (calc_forces_Ps_loc.jl:13-71)
//     F_a = sum_{G != 0} Re( i G V_sp(G) conj(rho(G)) e^{-i G.tau_a} ),  rho(G) = fft(rho)/N,
//     one CTA per (atom, chunk of the density sphere), partial sums reduced in
//     a fixed order (FP64, deterministic).
//   nonlocal (calc_forces_Ps_nloc.jl:291-411, GTH)
//     F_a += 2 w_s Re( h_ij conj(B_i,s) dB_j,s ) over the (i, j, h_ij) pairs of atom a,
//     B = betaNL' psi, dB = (i g betaNL)' psi = -i betaNL' (g o psi): psi is
//     scaled by each Cartesian component of g = G + k and the same projection
//     GEMM as op_V_Ps_nloc runs on it (no 3 x Ngw x NbetaNL dbetaNL array).
// The ion-ion (Ewald) force is host set-up arithmetic and stays with the caller.
#include <algorithm>
#include <vector>

#include "../../include/pwb200.h"
#include "pw_launch.h"

struct pw_ctx;
int pwk_fail(pw_ctx *c, int code, const char *msg);
int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out);
cudaStream_t pwk_stream(pw_ctx *c);
int pwk_device(const pw_ctx *c);
int pwk_ngw(const pw_ctx *c, int ik);
int pwk_nkpt(const pw_ctx *c);
void pwk_count_launches(pw_ctx *c, int n);
int pwk_density_to_G(pw_ctx *c, const double *rho, const double2 **rhoG, int *Ng);
int pwk_beta_dot(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, double2 *out);
int pwk_force_local_tables(pw_ctx *c, const double **G, const double **V, int *nsp, int *ng);
int pwk_force_nonlocal_tables(pw_ctx *c, int ik, const double **gk, const int **atom_rows, int *natoms, const int **rowptr,
                              const int **col, const double **val, int *nbeta);
int pwk_grid_points(const pw_ctx *c, size_t *N);

#define RK(x)                      \
    do {                           \
        int s_ = (x);              \
        if (s_ != 0) return s_;    \
    } while (0)
#define CKF(c, x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, #x " failed"); \
    } while (0)

namespace pwk {
namespace frc {

constexpr int LOC_CHUNK = 8192;   // density-sphere entries per CTA of the local force
constexpr int LOC_THREADS = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// part[(a * nchunk + chunk) * 3 + d]: this CTA's share of F_a
__global__ void __launch_bounds__(LOC_THREADS)
k_force_loc(const double *__restrict__ G, const double *__restrict__ V, int ng, const double2 *__restrict__ rhoG,
            double invN, const double *__restrict__ pos, const int *__restrict__ species, int nchunk,
            double *__restrict__ part) {
    __shared__ double red[3][LOC_THREADS / 32];
    const int a = blockIdx.y, chunk = blockIdx.x;
    const double tx = pos[3 * a], ty = pos[3 * a + 1], tz = pos[3 * a + 2];
    const double *Vs = V + (size_t)species[a] * ng;
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    const int g0 = chunk * LOC_CHUNK, g1 = min(ng, g0 + LOC_CHUNK);
    for (int g = max(g0, 1) + threadIdx.x; g < g1; g += LOC_THREADS) {   // G = 0 (first entry) skipped
        const double gx = G[3 * g], gy = G[3 * g + 1], gz = G[3 * g + 2];
        const double2 r = rhoG[g];
        const double v = Vs[g] * invN;
        // c = V conj(rho(G)); Re(i c e^{-i G.tau}) = Re(c) sin(G.tau) - Im(c) cos(G.tau)
        const double cr = v * r.x, ci = -v * r.y;
        double sn, cs;
        sincos(gx * tx + gy * ty + gz * tz, &sn, &cs);
        const double w = cr * sn - ci * cs;
        f0 += gx * w;
        f1 += gy * w;
        f2 += gz * w;
    }
    f0 = warp_sum(f0);
    f1 = warp_sum(f1);
    f2 = warp_sum(f2);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wp] = f0;
        red[1][wp] = f1;
        red[2][wp] = f2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int i = 0; i < LOC_THREADS / 32; ++i) s += red[threadIdx.x][i];
        part[((size_t)a * nchunk + chunk) * 3 + threadIdx.x] = s;
    }
}

__global__ void k_force_sum(const double *__restrict__ part, int natoms, int nchunk, double *__restrict__ F) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * natoms) return;
    const int a = t / 3, d = t - 3 * a;
    double s = 0.0;
    for (int c = 0; c < nchunk; ++c) s += part[((size_t)a * nchunk + c) * 3 + d];
    F[t] = s;
}

// psi_d[:, b] = g_d o psi[:, b] for d = 0, 1, 2 (three blocks of ld x nb)
template <typename T>
__global__ void k_scale_by_g(const Cx<T> *__restrict__ psi, int64_t ld, int ngw, int nb, const double *__restrict__ gk,
                             Cx<T> *__restrict__ out) {
    const size_t total = (size_t)ngw * nb;
    const size_t blk = (size_t)ld * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / ngw), g = (int)(t - (size_t)b * ngw);
        const Cx<T> p = psi[(size_t)b * ld + g];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T s = (T)gk[3 * g + d];
            out[d * blk + (size_t)b * ld + g] = cmake(p.x * s, p.y * s);
        }
    }
}

// One warp per atom: F_a[d] = sum over the atom's rows i and their
// coefficients (j, h) of sum_s 2 w_s Re(h conj(B[i,s]) dB_d[j,s]),
// dB_d = -i P_d with P_d = betaNL' (g_d o psi).
__global__ void k_force_nl(const int *__restrict__ atom_rows, int natoms, const int *__restrict__ rowptr,
                           const int *__restrict__ col, const double *__restrict__ val, const double2 *__restrict__ B,
                           const double2 *__restrict__ Pd, int nbeta, int nb, const double *__restrict__ w,
                           double *__restrict__ F) {
    const int lane = threadIdx.x & 31;
    const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (a >= natoms) return;
    const size_t blk = (size_t)nbeta * nb;
    double f[3] = {0.0, 0.0, 0.0};
    for (int i = atom_rows[a]; i < atom_rows[a + 1]; ++i) {
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const int j = col[e];
            const double h = val[e];
            for (int s = lane; s < nb; s += 32) {
                const double2 bi = B[(size_t)s * nbeta + i];
                const double ws = 2.0 * w[s] * h;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double2 p = Pd[d * blk + (size_t)s * nbeta + j];
                    // dB = -i p = (p.y, -p.x);  Re(conj(bi) dB) = bi.x p.y - bi.y p.x
                    f[d] += ws * (bi.x * p.y - bi.y * p.x);
                }
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double v = warp_sum(f[d]);
        if (lane == 0) F[3 * a + d] = v;
    }
}

}  // namespace frc
}  // namespace pwk

using namespace pwk;
using namespace pwk::frc;

extern "C" int pw_forces_local(pw_ctx *c, const double *rho, int natoms, const double *pos, const int32_t *species,
                               double *F) {
    if (!c) return PW_ERR_ARG;
    if (!rho || natoms <= 0 || !pos || !species || !F) return pwk_fail(c, PW_ERR_ARG, "bad pw_forces_local arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    const double *G = nullptr, *V = nullptr;
    int nsp = 0, ng = 0;
    RK(pwk_force_local_tables(c, &G, &V, &nsp, &ng));
    for (int a = 0; a < natoms; ++a)
        if (species[a] < 0 || species[a] >= nsp) return pwk_fail(c, PW_ERR_ARG, "species index out of range");
    const double2 *rhoG = nullptr;
    int ngd = 0;
    RK(pwk_density_to_G(c, rho, &rhoG, &ngd));
    if (ngd != ng) return pwk_fail(c, PW_ERR_STATE, "density sphere changed since pw_set_force_tables");
    cudaStream_t st = pwk_stream(c);
    const int nchunk = (ng + LOC_CHUNK - 1) / LOC_CHUNK;
    double *dpos = nullptr, *part = nullptr, *dF = nullptr;
    int *dsp = nullptr;
    RK(pwk_scratch(c, SL_FRC_A, (size_t)3 * natoms * sizeof(double), (void **)&dpos));
    RK(pwk_scratch(c, SL_FRC_B, (size_t)natoms * sizeof(int), (void **)&dsp));
    RK(pwk_scratch(c, SL_FRC_C, (size_t)natoms * nchunk * 3 * sizeof(double) + 3 * natoms * sizeof(double), (void **)&part));
    dF = part + (size_t)natoms * nchunk * 3;
    CKF(c, cudaMemcpyAsync(dpos, pos, (size_t)3 * natoms * sizeof(double), cudaMemcpyHostToDevice, st));
    CKF(c, cudaMemcpyAsync(dsp, species, (size_t)natoms * sizeof(int), cudaMemcpyHostToDevice, st));
    size_t N = 0;   // grid points: rho(G) = fft(rho) / N
    RK(pwk_grid_points(c, &N));
    k_force_loc<<<dim3(nchunk, natoms), LOC_THREADS, 0, st>>>(G, V, ng, rhoG, 1.0 / (double)N, dpos, dsp, nchunk, part);
    CKF(c, cudaGetLastError());
    k_force_sum<<<(3 * natoms + 127) / 128, 128, 0, st>>>(part, natoms, nchunk, dF);
    CKF(c, cudaGetLastError());
    CKF(c, cudaMemcpyAsync(F, dF, (size_t)3 * natoms * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKF(c, cudaStreamSynchronize(st));
    pwk_count_launches(c, 2);
    return PW_OK;
}

extern "C" int pw_forces_nonlocal(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, const double *w,
                                  double *F) {
    if (!c) return PW_ERR_ARG;
    if (dtype != PW_C128 && dtype != PW_C64) return pwk_fail(c, PW_ERR_ARG, "unknown dtype");
    if (ik < 0 || ik >= pwk_nkpt(c)) return pwk_fail(c, PW_ERR_ARG, "bad k-point index");
    const int ngw = pwk_ngw(c, ik);
    if (!psi || !w || !F || nb <= 0 || ld < ngw) return pwk_fail(c, PW_ERR_ARG, "bad pw_forces_nonlocal arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    const double *gk = nullptr, *val = nullptr;
    const int *atom_rows = nullptr, *rowptr = nullptr, *col = nullptr;
    int natoms = 0, nbeta = 0;
    RK(pwk_force_nonlocal_tables(c, ik, &gk, &atom_rows, &natoms, &rowptr, &col, &val, &nbeta));
    cudaStream_t st = pwk_stream(c);
    const size_t es = dtype == PW_C128 ? sizeof(double2) : sizeof(float2);
    const size_t blk = (size_t)nbeta * nb;
    char *psid = nullptr;
    double2 *B = nullptr, *Pd = nullptr;
    double *dw = nullptr, *dF = nullptr;
    RK(pwk_scratch(c, SL_FRC_A, 3 * (size_t)ld * nb * es, (void **)&psid));
    RK(pwk_scratch(c, SL_FRC_B, 4 * blk * sizeof(double2), (void **)&B));
    RK(pwk_scratch(c, SL_FRC_C, ((size_t)nb + 3 * natoms) * sizeof(double), (void **)&dw));
    Pd = B + blk;
    dF = dw + nb;
    CKF(c, cudaMemcpyAsync(dw, w, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, st));
    const int nblk = (int)std::min<size_t>(148 * 16, ((size_t)ngw * nb + 255) / 256);
    if (dtype == PW_C128)
        k_scale_by_g<double><<<nblk, 256, 0, st>>>((const double2 *)psi, ld, ngw, nb, gk, (double2 *)psid);
    else
        k_scale_by_g<float><<<nblk, 256, 0, st>>>((const float2 *)psi, ld, ngw, nb, gk, (float2 *)psid);
    CKF(c, cudaGetLastError());
    RK(pwk_beta_dot(c, ik, dtype, psi, ld, nb, B));
    for (int d = 0; d < 3; ++d) RK(pwk_beta_dot(c, ik, dtype, psid + (size_t)d * ld * nb * es, ld, nb, Pd + d * blk));
    k_force_nl<<<(natoms + 7) / 8, 256, 0, st>>>(atom_rows, natoms, rowptr, col, val, B, Pd, nbeta, nb, dw, dF);
    CKF(c, cudaGetLastError());
    CKF(c, cudaMemcpyAsync(F, dF, (size_t)3 * natoms * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKF(c, cudaStreamSynchronize(st));
    pwk_count_launches(c, 2);
    return PW_OK;
}
