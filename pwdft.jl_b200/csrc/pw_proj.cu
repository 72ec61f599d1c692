// Projector construction on the device: betaNL[ik] of the PsPotNL
// constructor (PsPotNL.jl:16-77) for GTH pseudopotentials,
//   beta[g, col] = (-i)^l Y_lm(G+k) p_{l,i}(|G+k|) e^{-i (G+k).tau_atom},
// with the radial projectors of eval_proj_G (PsPot_GTH.jl:338-391) and the
// real spherical harmonics of Ylm_real (Ylm_real.jl:5-107), one thread per
// (G+k, column), FP64.  The column table (atom, l, m, radial index, r_l and
// the normalisation 4 pi^(5/4) sqrt(2^(l+1) r_l^(2l+3) / Omega)) is the
// host's, in the reference's (atom, l, m, iprj) order.
#include <cmath>

#include "pw_launch.h"

namespace pwk {

__device__ double ylm_real(int l, int m, double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    const double ct = r < 1e-9 ? 0.0 : z / r;
    double phi;
    if (x > 1e-9)
        phi = atan(y / x);
    else if (x < -1e-9)
        phi = atan(y / x) + M_PI;
    else
        phi = y >= 0.0 ? M_PI / 2 : -M_PI / 2;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    switch (l * 10 + (m + 3)) {
        case 3: return 0.5 * sqrt(1.0 / M_PI);
        case 12: return 0.5 * sqrt(3.0 / M_PI) * st * sin(phi);
        case 13: return 0.5 * sqrt(3.0 / M_PI) * ct;
        case 14: return 0.5 * sqrt(3.0 / M_PI) * st * cos(phi);
        case 21: return sqrt(15.0 / 16.0 / M_PI) * st * st * sin(2 * phi);
        case 22: return sqrt(15.0 / 4.0 / M_PI) * ct * st * sin(phi);
        case 23: return 0.25 * sqrt(5.0 / M_PI) * (3.0 * ct * ct - 1.0);
        case 24: return sqrt(15.0 / 4.0 / M_PI) * ct * st * cos(phi);
        case 25: return sqrt(15.0 / 16.0 / M_PI) * st * st * cos(2 * phi);
        case 30: return 0.25 * sqrt(35.0 / 2.0 / M_PI) * st * st * st * sin(3 * phi);
        case 31: return 0.25 * sqrt(105.0 / M_PI) * st * st * ct * sin(2 * phi);
        case 32: return 0.25 * sqrt(21.0 / 2.0 / M_PI) * st * (5.0 * ct * ct - 1.0) * sin(phi);
        case 33: return 0.25 * sqrt(7.0 / M_PI) * (5.0 * ct * ct * ct - 3.0 * ct);
        case 34: return 0.25 * sqrt(21.0 / 2.0 / M_PI) * st * (5.0 * ct * ct - 1.0) * cos(phi);
        case 35: return 0.25 * sqrt(105.0 / M_PI) * st * st * ct * cos(2 * phi);
        case 36: return 0.25 * sqrt(35.0 / 2.0 / M_PI) * st * st * st * cos(3 * phi);
    }
    return 0.0;
}

// radial polynomial of eval_proj_G without the normalisation (i 1-based)
__device__ double gth_radial(int l, int i, double Gm, double rc) {
    const double x = (Gm * rc) * (Gm * rc);
    const double e = exp(-0.5 * x);
    switch (l * 10 + i) {
        case 1: return e;
        case 2: return 2.0 / sqrt(15.0) * e * (3.0 - x);
        case 3: return (4.0 / 3.0) / sqrt(105.0) * e * (15.0 - 10.0 * x + x * x);
        case 11: return e * Gm / sqrt(3.0);
        case 12: return 2.0 / sqrt(105.0) * e * Gm * (5.0 - x);
        case 13: return (4.0 / 3.0) / sqrt(1155.0) * e * Gm * (35.0 - 14.0 * x + x * x);
        case 21: return e * Gm * Gm / sqrt(15.0);
        case 22: return (2.0 / 3.0) / sqrt(105.0) * e * Gm * Gm * (7.0 - x);
        case 31: return Gm * Gm * Gm * e / sqrt(105.0);
    }
    return 0.0;
}

__global__ void k_build_beta(const double *__restrict__ gk, int ngw, const ProjCol *__restrict__ cols, int ncol,
                             const double *__restrict__ pos, double2 *__restrict__ beta) {
    const size_t total = (size_t)ngw * ncol;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t / ngw), g = (int)(t - (size_t)c * ngw);
        const ProjCol pc = cols[c];
        const double x = gk[3 * g], y = gk[3 * g + 1], z = gk[3 * g + 2];
        const double Gm = sqrt(x * x + y * y + z * z);
        const double a = pc.pref * ylm_real(pc.l, pc.m, x, y, z) * gth_radial(pc.l, pc.i, Gm, pc.rc);
        const double gx = x * pos[3 * pc.atom] + y * pos[3 * pc.atom + 1] + z * pos[3 * pc.atom + 2];
        double sn, cs;
        sincos(gx, &sn, &cs);
        // a e^{-i gx} (cs - i sn), times (-i)^l
        double re = a * cs, im = -a * sn;
        for (int k = 0; k < pc.l; ++k) {
            const double t2 = re;
            re = im;
            im = -t2;
        }
        beta[t] = make_double2(re, im);
    }
}

cudaError_t launch_build_beta(const double *gk, int ngw, const ProjCol *cols, int ncol, const double *pos, double2 *beta,
                              cudaStream_t st) {
    size_t b = ((size_t)ngw * ncol + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    k_build_beta<<<(int)(b < 1 ? 1 : b), 256, 0, st>>>(gk, ngw, cols, ncol, pos, beta);
    return cudaGetLastError();
}

}  // namespace pwk
