"""Shared-memory layouts of the FP32 fused line FFTs (pw_fft_fused.cuh,
pw_fft_kernels.cu), checked on the CPU with the header's own constexpr
functions (compiled by nvcc into a host-only program):

  fp_pos / fp_xs   element positions: injective, inside the line stride
  LaneMap          whole lines per half-warp: every load and store of both
                   stages of the 75- and 120-point lines (line stride N)
                   touches each bank pair of a half-warp once, where the
                   packed lane order conflicts
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
// LaneMap<NBF, G>: "LM NBF G ROUNDS" then (t lane ok line j) for every slot
template <int NBF, int G> void lanes() {
    using LM = pwf::LaneMap<NBF, G>;
    std::printf("LM %d %d %d", NBF, G, LM::ROUNDS);
    for (int t = 0; t < LM::ROUNDS; ++t)
        for (int lane = 0; lane < 32; ++lane) {
            int line = -1, j = -1;
            const bool ok = LM::at(lane, t, G, line, j);
            std::printf(" %d,%d,%d,%d,%d", t, lane, ok ? 1 : 0, line, j);
        }
    std::printf("\n");
}
template <int N> void dump() {
    constexpr int R0 = pwf::FPlan<N>::r(0);
    constexpr int R1 = pwf::FPlan<N>::nst == 2 ? pwf::FPlan<N>::r(1) : 1;
    std::printf("N %d G %d XS %d R0 %d R1 %d\n", N, pwf::fp_group<N>(), pwf::fp_xs<N>(), R0, R1);
    std::printf("POS");
    for (int x = 0; x < N; ++x) std::printf(" %d", pwf::fp_pos<N>(x));
    std::printf("\nTW");
    for (int i = 0; i < N; ++i) std::printf(" %d", pwf::tw_src<N>(i));
    std::printf("\n");
    lanes<N / R0, pwf::fp_group<N>()>();
    lanes<N / R1, pwf::fp_group<N>()>();
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
    for i in range(0, len(out) - 4, 5):
        f = out[i].split()
        N = int(f[1])
        res[N] = dict(G=int(f[3]), XS=int(f[5]), R0=int(f[7]), R1=int(f[9]),
                      pos=[int(v) for v in out[i + 1].split()[1:]], tw=[int(v) for v in out[i + 2].split()[1:]],
                      lanes={})
        for k in (3, 4):
            g = out[i + k].split()
            slots = [tuple(int(v) for v in x.split(",")) for x in g[4:]]
            res[N]["lanes"][int(g[1])] = dict(G=int(g[2]), rounds=int(g[3]), slots=slots)
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


def stage_patterns(L, nbf, packed=False):
    """Per warp instruction of the two stages of a warp group's lines: element
    indices within the lines (line stride XS) for every (round, r)."""
    N, XS, R0 = len(L["pos"]), L["XS"], L["R0"]
    lm = L["lanes"][nbf]
    R = N // nbf
    out = []
    rounds = (lm["G"] * nbf + 31) // 32 if packed else lm["rounds"]
    for t in range(rounds):
        slots = []
        for lane in range(32):
            if packed:
                i = lane + 32 * t
                slots.append((i // nbf, i % nbf) if i < lm["G"] * nbf else None)
            else:
                _, _, ok, line, j = lm["slots"][t * 32 + lane]
                slots.append((line, j) if ok else None)
        for r in range(R):
            if nbf == N // R0:      # first stage: reads j + nbf r, writes R0 j + r
                ld = [s[0] * XS + L["pos"][s[1] + nbf * r] if s else None for s in slots]
                st = [s[0] * XS + L["pos"][R0 * s[1] + r] if s else None for s in slots]
            else:                   # second stage: reads and writes j + R0 r
                ld = st = [s[0] * XS + L["pos"][s[1] + R0 * r] if s else None for s in slots]
            out += [ld, st]
    return out


def wavefronts_lanes(act):
    """wavefronts() with explicit lane numbers (idle lanes left out)."""
    tot = 0
    for half in (0, 1):
        h = [x for k, x in act if (k >= 16) == bool(half)]
        if h:
            banks = {}
            for x in h:
                banks.setdefault(x % 16, set()).add(x)
            tot += max(len(v) for v in banks.values())
    return tot


def test_line_stages_conflict_free(layouts):
    for N in (75, 120):
        L = layouts[N]
        for nbf in L["lanes"]:
            got = ideal = packed = 0
            for a in stage_patterns(L, nbf):
                act = [(k, x) for k, x in enumerate(a) if x is not None]
                got += wavefronts_lanes(act)
                ideal += (1 if any(k < 16 for k, _ in act) else 0) + (1 if any(k >= 16 for k, _ in act) else 0)
            for a in stage_patterns(L, nbf, packed=True):
                packed += wavefronts_lanes([(k, x) for k, x in enumerate(a) if x is not None])
            assert got == ideal, (N, nbf, got, ideal)
            assert got <= packed, (N, nbf, got, packed)
        # every slot of a group is taken exactly once over the rounds
        for nbf, lm in L["lanes"].items():
            seen = [(line, j) for t, lane, ok, line, j in lm["slots"] if ok]
            assert sorted(seen) == [(l, j) for l in range(lm["G"]) for j in range(nbf)], (N, nbf)


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
