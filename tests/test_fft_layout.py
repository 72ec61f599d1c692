"""Shared-memory layouts of the FP32 fused line FFTs (pw_fft_fused.cuh,
pw_fft_kernels.cu), checked on the CPU with the header's own constexpr
functions (compiled by nvcc into a host-only program):

  fp_pos / fp_xs   padded element positions: injective, inside the line
                   stride; on the 120-point lines every first-stage access
                   pattern of a warp touches each bank pair of a half-warp
                   once and the second stage at most twice
  tw_src           the shared twiddle table holds exp(-2 pi i m / R0) then
                   the stage-1 twiddles at (r, j), N entries
  zrow             the z-tile row stride = lines per warp group (mod 16)
                   tiles the 16 bank pairs for the line FFTs' lane pattern
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pwdft.jl_b200", "csrc")

PROG = r'''
#include <cstdio>
#include "pw_fft_fused.cuh"
template <int N> void dump() {
    constexpr int R0 = pwf::FPlan<N>::r(0);
    constexpr int R1 = pwf::FPlan<N>::nst == 2 ? pwf::FPlan<N>::r(1) : 1;
    std::printf("N %d G %d XS %d R0 %d R1 %d\n", N, pwf::fp_group<N>(), pwf::fp_xs<N>(), R0, R1);
    std::printf("POS");
    for (int x = 0; x < N; ++x) std::printf(" %d", pwf::fp_pos<N>(x));
    std::printf("\nTW");
    for (int i = 0; i < N; ++i) std::printf(" %d", pwf::tw_src<N>(i));
    std::printf("\n");
}
int main() { dump<27>(); dump<75>(); dump<120>(); return 0; }
'''


@pytest.fixture(scope="module")
def layouts(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("layout")
    src = d / "dump.cu"
    src.write_text(PROG)
    exe = str(d / "dump")
    subprocess.run(["nvcc", "-std=c++17", "-I", CSRC, str(src), "-o", exe], check=True, capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    res = {}
    for i in range(0, len(out) - 2, 3):
        f = out[i].split()
        N = int(f[1])
        res[N] = dict(G=int(f[3]), XS=int(f[5]), R0=int(f[7]), R1=int(f[9]),
                      pos=[int(v) for v in out[i + 1].split()[1:]], tw=[int(v) for v in out[i + 2].split()[1:]])
    return res


def wavefronts(addrs):
    """8-byte shared-memory accesses of one warp instruction: per half-warp,
    the largest number of distinct words on one bank pair."""
    tot = 0
    for h in (addrs[:16], addrs[16:32]):
        if h:
            banks = {}
            for a in h:
                banks.setdefault(a % 16, set()).add(a)
            tot += max(len(v) for v in banks.values())
    return tot


def test_positions_fit_and_are_injective(layouts):
    for N, L in layouts.items():
        assert len(set(L["pos"])) == N and max(L["pos"]) < L["XS"], N
        if N != 120:
            assert L["pos"] == list(range(N)) and L["XS"] == N


def test_120_first_stage_conflict_free(layouts):
    L = layouts[120]
    G, XS, R0, R1, pos = L["G"], L["XS"], L["R0"], L["R1"], L["pos"]
    ideal = got1 = got2 = 0
    for r in range(R0):                      # stage-0 outputs x = R0 j + r, lane (line, j)
        ids = list(range(G * R1))
        a = [(i // R1) * XS + pos[(i % R1) * R0 + r] for i in ids]
        got1 += wavefronts(a)
        ideal += (len(a) + 15) // 16
    assert got1 == ideal
    for r in range(R1):                      # stage-1 inputs x = j + R0 r, lane (line, j)
        for t in range((G * R0 + 31) // 32):
            ids = [i for i in range(32 * t, 32 * t + 32) if i < G * R0]
            a = [(i // R0) * XS + pos[(i % R0) + R0 * r] for i in ids]
            assert wavefronts(a) <= 2 * ((len(a) + 15) // 16)
            got2 += wavefronts(a)
    # the unpadded stride-120 layout: 8-way conflicts in stage 0
    bad = sum(wavefronts([(i // R1) * 120 + (i % R1) * R0 + r for i in range(G * R1)]) for r in range(R0))
    assert bad >= 7 * ideal


def test_twiddle_table(layouts):
    for N, L in layouts.items():
        tw = L["tw"]
        assert len(tw) == N and all(0 <= m < N for m in tw)
        if L["R1"] == 1:
            assert tw == list(range(N))
            continue
        R0, R1 = L["R0"], L["R1"]
        assert tw[:R0] == [m * (N // R0) for m in range(R0)]
        for r in range(1, R1):
            for j in range(R0):
                assert tw[R0 + (r - 1) * R0 + j] == r * j


def test_z_tile_stride(layouts):
    src = open(os.path.join(CSRC, "pw_fft_kernels.cu")).read()
    assert re.search(r"return G >= 16 \? \(Cg \| 1\) : Cg \+ \(\(G - Cg\) % 16 \+ 16\) % 16;", src)
    for N in (75, 120):
        G = layouts[N]["G"]
        for Cg in (38, 50, 64):
            Zs = Cg + ((G - Cg) % 16 + 16) % 16
            assert Zs >= Cg and Zs % 16 == G % 16
            # lane (line = id % G, j = id / G) reads word line + Zs j
            assert wavefronts([(i % G) + Zs * (i // G) for i in range(32)]) == 2
