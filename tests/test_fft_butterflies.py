"""Register DFTs of the line FFTs, compiled by nvcc into a host-only program
and compared with a direct DFT in double precision, both transform signs:

  - the FP32 butterflies (pw_fft.cuh, SmallDft<float, R>, R = 2, 3, 4, 5, 8),
    which run on the paired FP32 pipe of sm_100 (FFMA2 / FADD2 / FMUL2 with
    the products by +-i folded into swapped operand pairs); the host program
    takes the same lane-wise formulas with fmaf in place of the intrinsics;
  - the composite radices of the fused plans (pw_fft_fused.cuh, Dft<T, R>):
    9 = 3 x 3, 24 = 8 x 3, 25 = 5 x 5, 27 = 9 x 3 (Cooley-Tukey with
    compile-time roots) and 15 = 3 x 5 (prime-factor split, CRT output map),
    in FP32 and FP64, and the FP64 butterflies.

A wrong sign, lane swap, root or index map gives an O(1) error; rounding is
about 1e-7 (FP32) and 1e-16 (FP64) per unit of input.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pwdft.jl_b200", "csrc")

PROG = r'''
#include <cmath>
#include <cstdio>
#include <random>
#include "pw_fft_fused.cuh"
template <int R> double worst(float s) {
    std::mt19937 g(31 * R + (s > 0));
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    double w = 0.0;
    for (int trial = 0; trial < 2000; ++trial) {
        float2 v[R];
        double xr[R], xi[R];
        for (int n = 0; n < R; ++n) {
            v[n] = make_float2(U(g), U(g));
            xr[n] = v[n].x;
            xi[n] = v[n].y;
        }
        SmallDft<float, R>::run(v, s);
        for (int k = 0; k < R; ++k) {
            double ar = 0.0, ai = 0.0;
            for (int n = 0; n < R; ++n) {
                const double ang = (double)s * 2.0 * M_PI * (double)((n * k) % R) / R;
                ar += xr[n] * std::cos(ang) - xi[n] * std::sin(ang);
                ai += xr[n] * std::sin(ang) + xi[n] * std::cos(ang);
            }
            w = std::fmax(w, std::fmax(std::fabs(ar - v[k].x), std::fabs(ai - v[k].y)));
        }
    }
    return w;
}
// Dft<T, R> of the fused plans (composite radices with compile-time roots)
template <typename T, int R> double worst_dft(T s) {
    using C = Cx<T>;
    std::mt19937 g(97 * R + (s > 0) + 7 * (int)sizeof(T));
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    double w = 0.0;
    for (int trial = 0; trial < 500; ++trial) {
        C v[R];
        double xr[R], xi[R];
        for (int n = 0; n < R; ++n) {
            v[n] = cmake((T)U(g), (T)U(g));
            xr[n] = v[n].x;
            xi[n] = v[n].y;
        }
        pwf::Dft<T, R>::run(v, s, nullptr, 0);
        for (int k = 0; k < R; ++k) {
            double ar = 0.0, ai = 0.0;
            for (int n = 0; n < R; ++n) {
                const double ang = (double)s * 2.0 * M_PI * (double)((n * k) % R) / R;
                ar += xr[n] * std::cos(ang) - xi[n] * std::sin(ang);
                ai += xr[n] * std::sin(ang) + xi[n] * std::cos(ang);
            }
            w = std::fmax(w, std::fmax(std::fabs(ar - v[k].x), std::fabs(ai - v[k].y)));
        }
    }
    return w;
}
template <typename T> void composite(const char *tag) {
    for (T s : {(T)-1, (T)1})
        std::printf("%s %g %.3e %.3e %.3e %.3e %.3e %.3e %.3e %.3e %.3e %.3e\n", tag, (double)s, worst_dft<T, 2>(s),
                    worst_dft<T, 3>(s), worst_dft<T, 4>(s), worst_dft<T, 5>(s), worst_dft<T, 8>(s), worst_dft<T, 9>(s),
                    worst_dft<T, 15>(s), worst_dft<T, 24>(s), worst_dft<T, 25>(s), worst_dft<T, 27>(s));
}
int main() {
    for (float s : {-1.0f, 1.0f})
        std::printf("bfly %g %.3e %.3e %.3e %.3e %.3e\n", s, worst<2>(s), worst<3>(s), worst<4>(s), worst<5>(s), worst<8>(s));
    composite<float>("f32");
    composite<double>("f64");
    return 0;
}
'''


def test_register_dfts_match_direct_dft(tmp_path):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    src = tmp_path / "bfly.cu"
    src.write_text(PROG)
    exe = str(tmp_path / "bfly")
    subprocess.run(["nvcc", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", CSRC, str(src), "-o", exe],
                   check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = {}
    for line in out:
        if line.strip():
            f = line.split()
            rows[(f[0], float(f[1]))] = list(map(float, f[2:]))
    assert sorted(rows) == sorted((t, s) for t in ("bfly", "f32", "f64") for s in (-1.0, 1.0))
    for (tag, s), errs in rows.items():
        radices = (2, 3, 4, 5, 8) if tag == "bfly" else (2, 3, 4, 5, 8, 9, 15, 24, 25, 27)
        assert len(errs) == len(radices)
        for R, err in zip(radices, errs):
            tol = 1e-14 * R if tag == "f64" else 4e-7 * R
            assert err < tol, (tag, s, R, err)
