// update! and the energy reductions on the device (the step on either side
// of calc_rhoe / op_V_loc in KS_solve_SCF!):
//   Poisson_solve!   (Poisson_solve.jl:22-40):  rho(r) -> rho(G) on the density
//                    sphere (pruned forward FFT) -> 4 pi rho(G)/G^2 (G = 0 -> 0)
//                    -> V_H(r) = Re G_to_R
//   calc_Vxc_VWN!    (LDA_VWN_internal.jl:33-52, XC_funcs/XC_x_slater.jl,
//                    XC_funcs/XC_c_vwn.jl): eps_xc(r), V_xc(r)
//   calc_Vxc_PBE! / calc_epsxc_PBE! (GGA_PBE_internal.jl:29-145,
//                    XC_funcs/XC_x_pbe.jl, XC_c_pw.jl, XC_c_pbe.jl): grad rho
//                    by op_nabla (PWGrid.jl:351-375: i G rho(G) on the density
//                    sphere, three sphere-to-grid transforms), the pointwise
//                    functional, and div h by op_nabla_dot (PWGrid.jl:378-398:
//                    three grid-to-sphere transforms, i G . h(G), one back)
//   update!          (Hamiltonian.jl:510-545): V_tot = V_Ps_loc + V_H + V_xc,
//                    handed to op_V_loc as the context's V_loc
//   calc_E_local     (calc_energies.jl:245-333): E_Hartree, E_Ps_loc, E_xc
//   calc_E_kin / calc_E_Ps_nloc (calc_energies.jl:342-375, 7-58)
// All reductions are FP64 and deterministic (fixed block partials summed by
// one block).
#include <cmath>
#include <vector>

#include "../../include/pwb200.h"
#include "pw_fft.cuh"
#include "pw_launch.h"

int pwk_fail(pw_ctx *c, int code, const char *msg);
int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out);
cudaStream_t pwk_stream(pw_ctx *c);
int pwk_device(const pw_ctx *c);
void pwk_count_launches(pw_ctx *c, int n);
int pwk_density_launch(pw_ctx *c, pwk::FftLaunch *L, const double **G2, int *Ng, size_t *N);
int pwk_set_vloc_device(pw_ctx *c, const double *V, int nspin);
int pwk_projections(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, const double2 **P,
                    const double2 **P2, int *nbeta);
int pwk_ngw(const pw_ctx *c, int ik);
const double *pwk_gk2(const pw_ctx *c, int ik);
int pwk_xc(const pw_ctx *c, const double **G);
int pwk_symmetry(const pw_ctx *c, const int **isg, const double2 **ph, int *nshell, int *nsym);

namespace pwk {
namespace upd {

constexpr int RED_BLOCKS = 296;

// ------------------------------------------------------------ plane kernels
// real rho plane -> forward x-FFT -> active-x sub-plane -> forward y-FFT -> A
__global__ void __launch_bounds__(256)
k_plane_r2g(KPlan kp, FftDim dx, FftDim dy, const double2 *__restrict__ twx, const double2 *__restrict__ twy,
            const double *__restrict__ rho, double2 *__restrict__ A, int Jc) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int N1 = kp.N1, N2 = kp.N2, Nxa = kp.Nxa, Ncol = kp.Ncol;
    double2 *tx = reinterpret_cast<double2 *>(sm);
    double2 *ty = tx + N1;
    double2 *S = ty + N2;
    double2 *X = S + (size_t)Nxa * N2;
    const int kz = blockIdx.x;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[i];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[i];
    const double *rp = rho + (size_t)kz * N1 * N2;
    for (int j0 = 0; j0 < N2; j0 += Jc) {
        const int jc = min(Jc, N2 - j0);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = make_double2(rp[(size_t)j0 * N1 + i], 0.0);
        __syncthreads();
        fft_lines_w<double, 8>(X, dx, jc, 1, N1, tx, -1);
        for (int p = threadIdx.x; p < Nxa * jc; p += blockDim.x) {
            const int ia = p / jc, jl = p - ia * jc;
            S[ia * N2 + j0 + jl] = X[jl * N1 + kp.xa[ia]];
        }
        __syncthreads();
    }
    fft_lines_w<double, 8>(S, dy, Nxa, 1, N2, ty, -1);
    double2 *Ap = A + (size_t)kz * Ncol;
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) Ap[c] = S[kp.col_ia[c] * N2 + kp.col_j[c]];
}

// A -> inverse y-FFT -> inverse x-FFT -> out(r) = scale * Re
__global__ void __launch_bounds__(256)
k_plane_g2r(KPlan kp, FftDim dx, FftDim dy, const double2 *__restrict__ twx, const double2 *__restrict__ twy,
            const double2 *__restrict__ A, double *__restrict__ out, double scale, int Jc) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int N1 = kp.N1, N2 = kp.N2, Nxa = kp.Nxa, Ncol = kp.Ncol;
    double2 *tx = reinterpret_cast<double2 *>(sm);
    double2 *ty = tx + N1;
    double2 *S = ty + N2;
    double2 *X = S + (size_t)Nxa * N2;
    const int kz = blockIdx.x;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[i];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[i];
    for (int i = threadIdx.x; i < Nxa * N2; i += blockDim.x) S[i] = make_double2(0.0, 0.0);
    __syncthreads();
    const double2 *Ap = A + (size_t)kz * Ncol;
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
    __syncthreads();
    fft_lines_w<double, 8>(S, dy, Nxa, 1, N2, ty, +1);
    double *op = out + (size_t)kz * N1 * N2;
    for (int j0 = 0; j0 < N2; j0 += Jc) {
        const int jc = min(Jc, N2 - j0);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = make_double2(0.0, 0.0);
        __syncthreads();
        for (int p = threadIdx.x; p < Nxa * jc; p += blockDim.x) {
            const int ia = p / jc, jl = p - ia * jc;
            X[jl * N1 + kp.xa[ia]] = S[ia * N2 + j0 + jl];
        }
        __syncthreads();
        fft_lines_w<double, 8>(X, dx, jc, 1, N1, tx, +1);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) op[(size_t)j0 * N1 + i] = scale * X[i].x;
        __syncthreads();
    }
}

// VG[ig] = 4 pi rhoG[ig] / G2[ig]; the G = 0 entry (G2 == 0) is zeroed
__global__ void k_poisson_scale(double2 *g, const double *__restrict__ G2, int Ng) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Ng; i += gridDim.x * blockDim.x) {
        const double s = G2[i] > 0.0 ? 4.0 * M_PI / G2[i] : 0.0;
        g[i] = make_double2(g[i].x * s, g[i].y * s);
    }
}

// XC_x_slater + XC_c_vwn (spin-unpolarised), and V_tot = V_ps + V_H + V_xc
__global__ void k_vwn_vtot(const double *__restrict__ rho, const double *__restrict__ Vps, const double *__restrict__ VH,
                           double *__restrict__ Vxc, double *__restrict__ eps, double *__restrict__ Vtot, size_t N) {
    const double third = 1.0 / 3.0, pi34 = 0.6203504908994;
    const double a = 0.0310907, b = 3.72744, c = 12.9352, x0 = -0.10498;
    const double q = sqrt(4.0 * c - b * b);
    const double f1 = 2.0 * b / q, f2 = b * x0 / (x0 * x0 + b * x0 + c), f3 = 2.0 * (2.0 * x0 + b) / q;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const double r = rho[i];
        double ex = 0.0, vx = 0.0;
        if (r > 1e-10) {
            const double rs = pi34 / pow(r, third);
            const double f = -0.687247939924714, alpha = 2.0 / 3.0;
            ex = f * alpha / rs;
            vx = 4.0 / 3.0 * f * alpha / rs;
        }
        const double rs = pi34 / pow(r, third);
        const double rs12 = sqrt(rs);
        const double fx = rs + b * rs12 + c;
        const double qx = atan(q / (2.0 * rs12 + b));
        const double ec = a * (log(rs / fx) + f1 * qx - f2 * (log((rs12 - x0) * (rs12 - x0) / fx) + f3 * qx));
        const double tx = 2.0 * rs12 + b, tt = tx * tx + q * q;
        const double vc = ec - rs12 * a / 6.0 *
                                   (2.0 / rs12 - tx / fx - 4.0 * b / tt - f2 * (2.0 / (rs12 - x0) - tx / fx - 4.0 * (2.0 * x0 + b) / tt));
        Vxc[i] = vx + vc;
        eps[i] = ex + ec;
        Vtot[i] = Vps[i] + VH[i] + vx + vc;
    }
}

// ------------------------------------------------------------------ PBE
// XC_x_slater (energy and potential per particle)
__device__ inline void slater(double r, double &ex, double &vx) {
    ex = vx = 0.0;
    if (r > 1e-10) {
        const double rs = 0.6203504908994 / cbrt(r);
        const double f = -0.687247939924714, alpha = 2.0 / 3.0;
        ex = f * alpha / rs;
        vx = 4.0 / 3.0 * f * alpha / rs;
    }
}
// XC_c_pw: Perdew-Wang 92 correlation per particle
__device__ inline void c_pw(double r, double &ec, double &vc) {
    ec = vc = 0.0;
    if (r <= 1e-10) return;
    const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
    const double rs = 0.6203504908994 / cbrt(r);
    const double rs12 = sqrt(rs), rs32 = rs * rs12, rs2 = rs * rs;
    const double om = 2.0 * a * (b1 * rs12 + b2 * rs + b3 * rs32 + b4 * rs2);
    const double dom = 2.0 * a * (0.5 * b1 * rs12 + b2 * rs + 1.5 * b3 * rs32 + 2.0 * b4 * rs2);
    const double olog = log(1.0 + 1.0 / om);
    ec = -2.0 * a * (1.0 + a1 * rs) * olog;
    vc = -2.0 * a * (1.0 + 2.0 / 3.0 * a1 * rs) * olog - 2.0 / 3.0 * a * (1.0 + a1 * rs) * dom / (om * (om + 1.0));
}
// XC_x_pbe: gradient part of PBE exchange (energy density sx, v1x, v2x)
__device__ inline void x_pbe(double r, double g2, double &sx, double &v1x, double &v2x) {
    sx = v1x = v2x = 0.0;
    if (r <= 1e-6 || g2 <= 1e-10) return;
    const double third = 1.0 / 3.0, k = 0.804, mu = 0.2195149727645171;
    const double c1 = 0.75 / M_PI, c2 = 3.093667726280136, c5 = 4.0 * third;
    const double agrho = sqrt(g2);
    const double kf = c2 * cbrt(r);
    const double dsg = 0.5 / kf;
    const double s1 = agrho * dsg / r;
    const double s2 = s1 * s1;
    const double ds = -c5 * s1;
    const double f2 = 1.0 + s2 * mu / k;
    const double fx = k - k / f2;
    const double exunif = -c1 * kf;
    const double sx_s = exunif * fx;
    const double dfx = 2.0 * mu * s1 / (f2 * f2);
    v1x = sx_s + exunif * third * fx + exunif * dfx * ds;
    v2x = exunif * dfx * dsg / agrho;
    sx = sx_s * r;
}
// XC_c_pbe: gradient correction to PW92 correlation (sc, v1c, v2c)
__device__ inline void c_pbe(double r, double g2, double &sc, double &v1c, double &v2c) {
    sc = v1c = v2c = 0.0;
    if (r <= 1e-6 || g2 <= 1e-10) return;
    const double ga = 0.0310906908696548950, be = 0.06672455060314922;
    const double xkf = 1.919158292677513, xks = 1.128379167095513;
    const double rs = 0.6203504908994 / cbrt(r);
    double ec, vc;
    c_pw(r, ec, vc);
    const double kf = xkf / rs;
    const double ks = xks * sqrt(kf);
    const double t = sqrt(g2) / (2.0 * ks * r);
    const double expe = exp(-ec / ga);
    const double af = be / ga * (1.0 / (expe - 1.0));
    const double bf = expe * (vc - ec);
    const double y = af * t * t;
    const double d = 1.0 + y + y * y;
    const double xy = (1.0 + y) / d;
    const double qy = y * y * (2.0 + y) / (d * d);
    const double s1 = 1.0 + be / ga * t * t * xy;
    const double h0 = ga * log(s1);
    const double dh0 = be * t * t / s1 * (-7.0 / 3.0 * xy - qy * (af * bf / be - 7.0 / 3.0));
    const double ddh0 = be / (2.0 * ks * ks * r) * (xy - qy) / s1;
    sc = r * h0;
    v1c = h0 + dh0;
    v2c = ddh0;
}

// out[ig] = i G_d[ig] rhoG[ig]  (one Cartesian component of op_nabla)
__global__ void k_grad_G(const double2 *__restrict__ rhoG, const double *__restrict__ G, int d, double2 *__restrict__ out,
                         int Ng) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Ng; i += gridDim.x * blockDim.x) {
        const double gd = G[3 * i + d];
        const double2 v = rhoG[i];
        out[i] = make_double2(-gd * v.y, gd * v.x);
    }
}
// div[ig] (+)= G_d[ig] hG[ig]; last: div := i div (op_nabla_dot)
__global__ void k_div_acc(double2 *__restrict__ div, const double2 *__restrict__ hG, const double *__restrict__ G, int d,
                          int Ng, int first, int last) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Ng; i += gridDim.x * blockDim.x) {
        const double gd = G[3 * i + d];
        double2 a = first ? make_double2(0.0, 0.0) : div[i];
        a.x += gd * hG[i].x;
        a.y += gd * hG[i].y;
        div[i] = last ? make_double2(-a.y, a.x) : a;
    }
}
// pointwise PBE (GGA_PBE_internal.jl:39-50, 114-130): eps_xc, the local
// part of V_xc, and h = (v2x + v2c) grad rho written over grad rho
__global__ void k_pbe_point(const double *__restrict__ rho, double *__restrict__ gx, double *__restrict__ gy,
                            double *__restrict__ gz, double *__restrict__ Vxc, double *__restrict__ eps, size_t N) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const double r = rho[i];
        const double a = gx[i], b = gy[i], c = gz[i];
        const double g2 = a * a + b * b + c * c;
        double ex, vx, ec, vc, sx, v1x, v2x, sc, v1c, v2c;
        slater(r, ex, vx);
        c_pw(r, ec, vc);
        x_pbe(r, g2, sx, v1x, v2x);
        c_pbe(r, g2, sc, v1c, v2c);
        eps[i] = ex + ec + (r != 0.0 ? (sx + sc) / r : 0.0);
        Vxc[i] = vx + vc + v1x + v1c;
        const double v2 = v2x + v2c;
        gx[i] = v2 * a;
        gy[i] = v2 * b;
        gz[i] = v2 * c;
    }
}
// symmetrize_rhoe! (RhoeSymmetrizer.jl:153-228), one thread per orbit of
// the density sphere: rhosum = (1/nsym) sum_s rho(isg_s) conj(ph_s), then
// rho(isg_s) := rhosum ph_s in operation order (a later operation that hits
// the same G wins, as in the reference); written as the change delta(G).
__global__ void k_sym_orbits(const double2 *__restrict__ rhoG, const int *__restrict__ isg,
                             const double2 *__restrict__ ph, int nshell, int nsym, double2 *__restrict__ delta) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nshell) return;
    const int *ix = isg + (size_t)o * nsym;
    const double2 *p = ph + (size_t)o * nsym;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsym; ++s) {
        const double2 r = rhoG[ix[s]], q = p[s];
        re += r.x * q.x + r.y * q.y;
        im += r.y * q.x - r.x * q.y;
    }
    re /= nsym;
    im /= nsym;
    for (int s = 0; s < nsym; ++s) {
        const double2 r = rhoG[ix[s]], q = p[s];
        delta[ix[s]] = make_double2(re * q.x - im * q.y - r.x, re * q.y + im * q.x - r.y);
    }
}
__global__ void k_add(double *__restrict__ y, const double *__restrict__ x, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] += x[i];
}

// V_xc -= div h; V_tot = V_ps + V_H + V_xc
__global__ void k_pbe_vtot(double *__restrict__ Vxc, const double *__restrict__ dh, const double *__restrict__ Vps,
                           const double *__restrict__ VH, double *__restrict__ Vtot, size_t N) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const double v = Vxc[i] - dh[i];
        Vxc[i] = v;
        Vtot[i] = Vps[i] + VH[i] + v;
    }
}

// partial sums of  sum_i w_k(i) * x_k(i) * y_k(i)  for three products
__global__ void k_dot3(const double *__restrict__ x0, const double *__restrict__ y0, const double *__restrict__ x1,
                       const double *__restrict__ y1, const double *__restrict__ x2, const double *__restrict__ y2, size_t N,
                       double *__restrict__ part) {
    __shared__ double red[3][32];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        s0 += x0[i] * y0[i];
        s1 += x1[i] * y1[i];
        s2 += x2[i] * y2[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = s0;
        red[1][w] = s1;
        red[2][w] = s2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[threadIdx.x][i];
        part[blockIdx.x * 3 + threadIdx.x] = s;
    }
}

// E_kin partials: sum_b w_b sum_g |psi_bg|^2 Gk2_g (FP64 accumulation)
template <typename T>
__global__ void k_ekin(const Cx<T> *__restrict__ psi, int64_t ld, int Ngw, int nb, const double *__restrict__ Gk2,
                       const double *__restrict__ w, double *__restrict__ part) {
    __shared__ double red[32];
    double s = 0.0;
    const size_t total = (size_t)Ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int bnd = (int)(t / Ngw), g = (int)(t - (size_t)bnd * Ngw);
        const Cx<T> v = psi[(size_t)bnd * ld + g];
        s += w[bnd] * ((double)v.x * v.x + (double)v.y * v.y) * Gk2[g];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) a += red[i];
        part[blockIdx.x] = a;
    }
}

// E_nl partials: sum_b w_b Re sum_i conj(P_ib) (D P)_ib
__global__ void k_enl(const double2 *__restrict__ P, const double2 *__restrict__ P2, int nbeta, int nb,
                      const double *__restrict__ w, double *__restrict__ part) {
    __shared__ double red[32];
    double s = 0.0;
    const size_t total = (size_t)nbeta * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int bnd = (int)(t / nbeta);
        s += w[bnd] * (P[t].x * P2[t].x + P[t].y * P2[t].y);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) a += red[i];
        part[blockIdx.x] = a;
    }
}

}  // namespace upd
}  // namespace pwk

using namespace pwk;
using namespace pwk::upd;

#define RK(x)                       \
    do {                            \
        int s_ = (x);               \
        if (s_ != PW_OK) return s_; \
    } while (0)
#define CKU(c, x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, #x " failed"); \
    } while (0)

static size_t plane_smem(const FftLaunch &L) {
    return ((size_t)L.kp.N1 + L.kp.N2 + (size_t)L.kp.Nxa * L.kp.N2 + (size_t)L.Jc * L.kp.N1) * sizeof(double2);
}

// rho(r) (device, N) -> R_to_G(rho) on the density sphere (device, Ng),
// unnormalised (the reference's fft); A: the plane intermediate.
static int density_to_G(pw_ctx *c, const double *rho, FftLaunch &L, double2 **gout, double2 **Aout, int *Ngout,
                        size_t *Nout, const double **G2out) {
    const double *G2 = nullptr;
    int Ng = 0;
    size_t N = 0;
    RK(pwk_density_launch(c, &L, &G2, &Ng, &N));
    cudaStream_t st = pwk_stream(c);
    double2 *A = nullptr, *g = nullptr;
    RK(pwk_scratch(c, SL_UPD_A, (size_t)L.kp.N3 * L.kp.Ncol * sizeof(double2), (void **)&A));
    RK(pwk_scratch(c, SL_UPD_RHOG, (size_t)Ng * sizeof(double2), (void **)&g));
    const size_t smem = plane_smem(L);
    if (smem > 48 * 1024) {
        CKU(c, cudaFuncSetAttribute((const void *)k_plane_r2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CKU(c, cudaFuncSetAttribute((const void *)k_plane_g2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    k_plane_r2g<<<L.kp.N3, 256, smem, st>>>(L.kp, L.dx, L.dy, (const double2 *)L.twx, (const double2 *)L.twy, rho, A, L.Jc);
    CKU(c, cudaGetLastError());
    CKU(c, launch_zfwd<double>(L, A, g, g, Ng, 1, 0, st));  // sphere coefficients of R_to_G(rho)
    pwk_count_launches(c, 2);
    *gout = g;
    *Aout = A;
    *Ngout = Ng;
    *Nout = N;
    *G2out = G2;
    return PW_OK;
}

int pwk_density_to_G(pw_ctx *c, const double *rho, const double2 **rhoG, int *Ng) {
    FftLaunch L;
    double2 *g = nullptr, *A = nullptr;
    size_t N = 0;
    const double *G2 = nullptr;
    RK(density_to_G(c, rho, L, &g, &A, Ng, &N, &G2));
    *rhoG = g;
    return PW_OK;
}

// rho(r) (device, N) -> V_H(r) (device, N): Poisson_solve!
static int poisson(pw_ctx *c, const double *rho, double *VH) {
    FftLaunch L;
    const double *G2 = nullptr;
    int Ng = 0;
    size_t N = 0;
    double2 *A = nullptr, *g = nullptr;
    RK(density_to_G(c, rho, L, &g, &A, &Ng, &N, &G2));
    cudaStream_t st = pwk_stream(c);
    const size_t smem = plane_smem(L);
    k_poisson_scale<<<(Ng + 255) / 256, 256, 0, st>>>(g, G2, Ng);
    CKU(c, launch_zinv<double>(L, g, Ng, 1, A, st));
    k_plane_g2r<<<L.kp.N3, 256, smem, st>>>(L.kp, L.dx, L.dy, (const double2 *)L.twx, (const double2 *)L.twy, A, VH,
                                            1.0 / (double)N, L.Jc);
    CKU(c, cudaGetLastError());
    pwk_count_launches(c, 3);
    return PW_OK;
}

// sphere coefficients g (device, Ng; clobbered by the z pass) -> out(r) =
// Re G_to_R (the reference's ifft, 1/N)
static int sphere_to_R(pw_ctx *c, FftLaunch &L, const double2 *g, int Ng, size_t N, double *out) {
    cudaStream_t st = pwk_stream(c);
    double2 *A = nullptr;
    RK(pwk_scratch(c, SL_UPD_A, (size_t)L.kp.N3 * L.kp.Ncol * sizeof(double2), (void **)&A));
    CKU(c, launch_zinv<double>(L, g, Ng, 1, A, st));
    k_plane_g2r<<<L.kp.N3, 256, plane_smem(L), st>>>(L.kp, L.dx, L.dy, (const double2 *)L.twx, (const double2 *)L.twy, A,
                                                     out, 1.0 / (double)N, L.Jc);
    CKU(c, cudaGetLastError());
    pwk_count_launches(c, 2);
    return PW_OK;
}

// calc_Vxc_PBE! + calc_epsxc_PBE! (Nspin = 1): Vxc (N) and eps (N) from rho
static int pbe(pw_ctx *c, const double *rho, const double *G, double *Vxc, double *eps) {
    FftLaunch L;
    double2 *g = nullptr, *A = nullptr, *div = nullptr, *tmp = nullptr;
    int Ng = 0;
    size_t N = 0;
    const double *G2 = nullptr;
    RK(density_to_G(c, rho, L, &g, &A, &Ng, &N, &G2));
    cudaStream_t st = pwk_stream(c);
    double *grad = nullptr;
    RK(pwk_scratch(c, SL_UPD_GRAD, 3 * N * sizeof(double), (void **)&grad));
    RK(pwk_scratch(c, SL_UPD_DIVG, 2 * (size_t)Ng * sizeof(double2), (void **)&div));
    tmp = div + Ng;
    const int gb = (Ng + 255) / 256;
    // grad rho (op_nabla)
    for (int d = 0; d < 3; ++d) {
        k_grad_G<<<gb, 256, 0, st>>>(g, G, d, tmp, Ng);
        CKU(c, cudaGetLastError());
        pwk_count_launches(c, 1);
        RK(sphere_to_R(c, L, tmp, Ng, N, grad + d * N));
    }
    k_pbe_point<<<RED_BLOCKS, 256, 0, st>>>(rho, grad, grad + N, grad + 2 * N, Vxc, eps, N);
    CKU(c, cudaGetLastError());
    pwk_count_launches(c, 1);
    // div h (op_nabla_dot)
    for (int d = 0; d < 3; ++d) {
        RK(density_to_G(c, grad + d * N, L, &g, &A, &Ng, &N, &G2));
        k_div_acc<<<gb, 256, 0, st>>>(div, g, G, d, Ng, d == 0, d == 2);
        CKU(c, cudaGetLastError());
        pwk_count_launches(c, 1);
    }
    RK(sphere_to_R(c, L, div, Ng, N, grad));   // div h(r) over h_x, no longer needed
    return PW_OK;
}

extern "C" int pw_symmetrize_rhoe(pw_ctx *c, double *rho) {
    if (!c) return PW_ERR_ARG;
    if (!rho) return pwk_fail(c, PW_ERR_ARG, "NULL density");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    const int *isg = nullptr;
    const double2 *ph = nullptr;
    int nshell = 0, nsym = 0;
    if (pwk_symmetry(c, &isg, &ph, &nshell, &nsym) != PW_OK)
        return pwk_fail(c, PW_ERR_STATE, "symmetry tables are not set (pw_set_symmetry)");
    FftLaunch L;
    double2 *g = nullptr, *A = nullptr, *delta = nullptr;
    int Ng = 0;
    size_t N = 0;
    const double *G2 = nullptr;
    RK(density_to_G(c, rho, L, &g, &A, &Ng, &N, &G2));
    cudaStream_t st = pwk_stream(c);
    double *tmp = nullptr;
    RK(pwk_scratch(c, SL_UPD_DIVG, (size_t)Ng * sizeof(double2), (void **)&delta));
    RK(pwk_scratch(c, SL_UPD_GRAD, N * sizeof(double), (void **)&tmp));
    k_sym_orbits<<<(nshell + 127) / 128, 128, 0, st>>>(g, isg, ph, nshell, nsym, delta);
    CKU(c, cudaGetLastError());
    RK(sphere_to_R(c, L, delta, Ng, N, tmp));
    k_add<<<RED_BLOCKS, 256, 0, st>>>(rho, tmp, N);
    CKU(c, cudaGetLastError());
    pwk_count_launches(c, 2);
    return PW_OK;
}

extern "C" int pw_poisson(pw_ctx *c, const double *rho, double *VH) {
    if (!c) return PW_ERR_ARG;
    if (!rho || !VH) return pwk_fail(c, PW_ERR_ARG, "NULL density or potential");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    return poisson(c, rho, VH);
}

extern "C" int pw_update(pw_ctx *c, const double *rho, const double *Vps, double *VH, double *Vxc, double *E3) {
    if (!c) return PW_ERR_ARG;
    if (!rho || !Vps || !E3) return pwk_fail(c, PW_ERR_ARG, "NULL argument to pw_update");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    FftLaunch L;
    const double *G2 = nullptr;
    int Ng = 0;
    size_t N = 0;
    RK(pwk_density_launch(c, &L, &G2, &Ng, &N));
    cudaStream_t st = pwk_stream(c);
    double *vh = VH, *vxc = Vxc, *eps = nullptr, *vt = nullptr, *part = nullptr;
    if (!vh) RK(pwk_scratch(c, SL_UPD_VH, N * sizeof(double), (void **)&vh));
    if (!vxc) RK(pwk_scratch(c, SL_UPD_VXC, N * sizeof(double), (void **)&vxc));
    RK(pwk_scratch(c, SL_UPD_EPS, N * sizeof(double), (void **)&eps));
    RK(pwk_scratch(c, SL_UPD_VTOT, N * sizeof(double), (void **)&vt));
    RK(pwk_scratch(c, SL_UPD_RED, RED_BLOCKS * 3 * sizeof(double), (void **)&part));
    RK(poisson(c, rho, vh));
    const double *xcG = nullptr;
    if (pwk_xc(c, &xcG) == PW_XC_PBE) {
        RK(pbe(c, rho, xcG, vxc, eps));
        double *dh = nullptr;
        RK(pwk_scratch(c, SL_UPD_GRAD, 3 * N * sizeof(double), (void **)&dh));
        k_pbe_vtot<<<RED_BLOCKS, 256, 0, st>>>(vxc, dh, Vps, vh, vt, N);
    } else {
        k_vwn_vtot<<<RED_BLOCKS, 256, 0, st>>>(rho, Vps, vh, vxc, eps, vt, N);
    }
    CKU(c, cudaGetLastError());
    RK(pwk_set_vloc_device(c, vt, 1));
    k_dot3<<<RED_BLOCKS, 256, 0, st>>>(vh, rho, Vps, rho, eps, rho, N, part);
    CKU(c, cudaGetLastError());
    std::vector<double> h(RED_BLOCKS * 3);
    CKU(c, cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKU(c, cudaStreamSynchronize(st));
    double s[3] = {0, 0, 0};
    for (int b = 0; b < RED_BLOCKS; ++b)
        for (int k = 0; k < 3; ++k) s[k] += h[b * 3 + k];
    E3[0] = s[0];  // sum V_H rho   (E_Hartree = 0.5 * dVol * this)
    E3[1] = s[1];  // sum V_ps rho  (E_Ps_loc  = dVol * this)
    E3[2] = s[2];  // sum eps rho   (E_xc      = dVol * this)
    pwk_count_launches(c, 2);
    if (!std::isfinite(s[0]) || !std::isfinite(s[1]) || !std::isfinite(s[2]))
        return pwk_fail(c, PW_ERR_NAN, "non-finite local energy");
    return PW_OK;
}

extern "C" int pw_band_energies(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, const double *w,
                                double *E2) {
    if (!c) return PW_ERR_ARG;
    if (!psi || !w || !E2 || nb <= 0) return pwk_fail(c, PW_ERR_ARG, "bad pw_band_energies arguments");
    if (cudaSetDevice(pwk_device(c)) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t st = pwk_stream(c);
    double *dw = nullptr, *part = nullptr;
    RK(pwk_scratch(c, SL_BAND_W, (size_t)nb * sizeof(double), (void **)&dw));
    RK(pwk_scratch(c, SL_BAND_RED, 2 * RED_BLOCKS * sizeof(double), (void **)&part));
    CKU(c, cudaMemcpyAsync(dw, w, nb * sizeof(double), cudaMemcpyHostToDevice, st));
    const int Ngw = pwk_ngw(c, ik);
    if (dtype == PW_C128)
        k_ekin<double><<<RED_BLOCKS, 256, 0, st>>>((const double2 *)psi, ld, Ngw, nb, pwk_gk2(c, ik), dw, part);
    else
        k_ekin<float><<<RED_BLOCKS, 256, 0, st>>>((const float2 *)psi, ld, Ngw, nb, pwk_gk2(c, ik), dw, part);
    CKU(c, cudaGetLastError());
    const double2 *P = nullptr, *P2 = nullptr;
    int nbeta = 0;
    RK(pwk_projections(c, ik, dtype, psi, ld, nb, &P, &P2, &nbeta));
    if (nbeta > 0) {
        k_enl<<<RED_BLOCKS, 256, 0, st>>>(P, P2, nbeta, nb, dw, part + RED_BLOCKS);
        CKU(c, cudaGetLastError());
    } else {
        CKU(c, cudaMemsetAsync(part + RED_BLOCKS, 0, RED_BLOCKS * sizeof(double), st));
    }
    std::vector<double> h(2 * RED_BLOCKS);
    CKU(c, cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CKU(c, cudaStreamSynchronize(st));
    double ek = 0.0, en = 0.0;
    for (int b = 0; b < RED_BLOCKS; ++b) {
        ek += h[b];
        en += h[RED_BLOCKS + b];
    }
    E2[0] = 0.5 * ek;  // E_kin contribution of this k-point (weights included)
    E2[1] = en;        // E_Ps_nloc contribution
    pwk_count_launches(c, 2);
    if (!std::isfinite(ek) || !std::isfinite(en)) return pwk_fail(c, PW_ERR_NAN, "non-finite band energy");
    return PW_OK;
}
