"""FP32 butterflies of the line FFTs (pw_fft.cuh, SmallDft<float, R>), which
run on the paired FP32 pipe of sm_100 (FFMA2 / FADD2 / FMUL2 with the
products by +-i folded into swapped operand pairs).  The same lane-wise
formulas are compiled by nvcc into a host-only program (fmaf in place of the
paired intrinsics) and compared with a direct DFT in double precision for
R = 2, 3, 4, 5, 8 and both transform signs: a wrong sign or lane swap gives
an O(1) error, FP32 rounding about 1e-7.
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
#include "pw_fft.cuh"
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
int main() {
    for (float s : {-1.0f, 1.0f})
        std::printf("%g %.3e %.3e %.3e %.3e %.3e\n", s, worst<2>(s), worst<3>(s), worst<4>(s), worst<5>(s), worst<8>(s));
    return 0;
}
'''


def test_fp32_butterflies_match_direct_dft(tmp_path):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    src = tmp_path / "bfly.cu"
    src.write_text(PROG)
    exe = str(tmp_path / "bfly")
    subprocess.run(["nvcc", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", CSRC, str(src), "-o", exe],
                   check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [list(map(float, line.split())) for line in out if line.strip()]
    assert [r[0] for r in rows] == [-1.0, 1.0]
    for r in rows:
        for R, err in zip((2, 3, 4, 5, 8), r[1:]):
            assert err < 2e-6, (r[0], R, err)
