// Host-side basis construction: FFT grid order, G-sphere and per-k
// wavefunction sphere index maps.
//
// Bit-exactness with the reference (PWGrid.jl) rests on evaluating every
// floating-point expression in the reference's order with no fused
// multiply-add (this file is compiled with -ffp-contract=off):
//   G[a]  = (R[a,1]*gi + R[a,2]*gj) + R[a,3]*gk            PWGrid.jl:218-220
//   G2    = (G1*G1 + G2*G2) + G3*G3                        PWGrid.jl:221
//   Gk2   = ((G1+k1)^2 + (G2+k2)^2) + (G3+k3)^2            PWGrid.jl:308-311
// and on ordering the sphere with a stable sort on G2 (Julia's sortperm
// breaks ties by index, PWGrid.jl:232).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "../../include/pwb200.h"

namespace {

// fft_support.jl:2-45
bool allowed(long nr) {
    static const long factors[5] = {2, 3, 5, 7, 11};
    long mr = nr;
    long pwr[5] = {0, 0, 0, 0, 0};
    bool done = false;
    for (int i = 0; i < 5 && !done; ++i) {
        const long fac = factors[i];
        const long maxpwr = std::lround(std::log((double)mr) / std::log((double)fac)) + 1;
        for (long p = 0; p < maxpwr; ++p) {
            if (mr == 1) {
                done = true;
                break;
            }
            if (mr % fac == 0) {
                mr /= fac;
                pwr[i] += 1;
            }
        }
    }
    if (mr != 1) return false;
    return pwr[3] == 0 && pwr[4] == 0;
}

// PWGrid.jl:157-163
inline long mm_to_nn(long mm, long S) { return (2 * mm > S) ? mm - S : mm; }

template <typename F>
void for_each_grid_point(const int32_t *Ns, const double *R, F f) {
    const long N1 = Ns[0], N2 = Ns[1], N3 = Ns[2];
    long ip = 0;
    for (long k = 0; k < N3; ++k)
        for (long j = 0; j < N2; ++j)
            for (long i = 0; i < N1; ++i, ++ip) {
                const double gi = (double)mm_to_nn(i, N1);
                const double gj = (double)mm_to_nn(j, N2);
                const double gk = (double)mm_to_nn(k, N3);
                // R is column-major: R[a,c] = R[a + 3c]
                const double g1 = (R[0] * gi + R[3] * gj) + R[6] * gk;
                const double g2 = (R[1] * gi + R[4] * gj) + R[7] * gk;
                const double g3 = (R[2] * gi + R[5] * gj) + R[8] * gk;
                const double G2 = (g1 * g1 + g2 * g2) + g3 * g3;
                f(ip, g1, g2, g3, G2);
            }
}

}  // namespace

extern "C" int pw_good_fft_order(int n) {
    long nr = n;
    while (!allowed(nr) && nr <= 2049) ++nr;
    if (nr > 2049) return -1;
    return (int)nr;
}

extern "C" int pw_gvec_count(const int32_t *Ns, const double *recvecs, double ecutrho, int64_t *Ng) {
    if (!Ns || !recvecs || !Ng || Ns[0] <= 0 || Ns[1] <= 0 || Ns[2] <= 0) return PW_ERR_ARG;
    int64_t n = 0;
    for_each_grid_point(Ns, recvecs, [&](long, double, double, double, double G2) {
        if (0.5 * G2 <= ecutrho) ++n;
    });
    *Ng = n;
    return PW_OK;
}

extern "C" int pw_gvec_build(const int32_t *Ns, const double *recvecs, double ecutrho, int64_t Ng, double *G, double *G2,
                             int64_t *idx_g2r) {
    if (!Ns || !recvecs || !G || !G2 || !idx_g2r) return PW_ERR_ARG;
    std::vector<double> g1, g2, g3, gg;
    std::vector<int64_t> ip;
    g1.reserve(Ng);
    for_each_grid_point(Ns, recvecs, [&](long p, double a, double b, double c, double G2v) {
        if (0.5 * G2v <= ecutrho) {
            g1.push_back(a);
            g2.push_back(b);
            g3.push_back(c);
            gg.push_back(G2v);
            ip.push_back(p);
        }
    });
    if ((int64_t)gg.size() != Ng) return PW_ERR_ARG;
    std::vector<int64_t> perm(Ng);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t x, int64_t y) { return gg[x] < gg[y]; });
    for (int64_t i = 0; i < Ng; ++i) {
        const int64_t s = perm[i];
        G[3 * i + 0] = g1[s];
        G[3 * i + 1] = g2[s];
        G[3 * i + 2] = g3[s];
        G2[i] = gg[s];
        idx_g2r[i] = ip[s];
    }
    return PW_OK;
}

extern "C" int pw_gvecw_build(int64_t Ng, const double *G, const int64_t *idx_g2r, const double *kpt, double ecutwfc,
                              int64_t *Ngw, int64_t *idx_gw2g, int64_t *idx_gw2r, double *Gk2) {
    if (!G || !idx_g2r || !kpt || !Ngw || !idx_gw2g || !idx_gw2r || !Gk2) return PW_ERR_ARG;
    int64_t n = 0;
    for (int64_t ig = 0; ig < Ng; ++ig) {
        const double a = G[3 * ig + 0] + kpt[0];
        const double b = G[3 * ig + 1] + kpt[1];
        const double c = G[3 * ig + 2] + kpt[2];
        double s = a * a + b * b;
        s = s + c * c;
        if (0.5 * s <= ecutwfc) {
            idx_gw2g[n] = ig;
            idx_gw2r[n] = idx_g2r[ig];
            Gk2[n] = s;
            ++n;
        }
    }
    *Ngw = n;
    return PW_OK;
}
