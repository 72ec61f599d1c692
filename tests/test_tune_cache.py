"""Host logic of the launch-parameter autotuner (pw_tune_cache.h, used by
pw_autotune in pw_tune.cu), compiled by g++ into a host-only program and
run on the CPU:

  cache    a choice appended under one key reads back field for field; other
           keys miss; the last matching line wins; lines without a tab or
           four numbers are skipped; a missing file or an empty path is a
           miss and appending to an empty path writes nothing
  key      the GPU name, grid, Ngw, active columns / x planes, nb, dtype and
           projector count all enter the key
  descent  one coordinate of the descent keeps the defaults unless a
           candidate is at least 0.5 % faster, skips failed candidates
           (negative time) and ends on the fastest value
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pwdft.jl_b200", "csrc")

PROG = r'''
#include <cstdio>
#include <map>
#include "pw_tune_cache.h"
using namespace pwk::tune;
static int fails = 0;
#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d: %s\n", __LINE__, #c); ++fails; } } while (0)
int main(int argc, char **argv) {
    const char *path = argv[1];
    const int Ns[3] = {75, 75, 75};
    const std::string k1 = cache_key("NVIDIA B200", Ns, 23871, 1005, 35, 160, 1, 320);
    const std::string k2 = cache_key("NVIDIA B200", Ns, 23871, 1005, 35, 160, 0, 320);
    CHECK(k1 != k2);
    CHECK(k1.find("gpu=NVIDIA B200") == 0 && k1.find("Ns=75x75x75") != std::string::npos &&
          k1.find("Ngw=23871") != std::string::npos && k1.find("Ncol=1005") != std::string::npos &&
          k1.find("Nxa=35") != std::string::npos && k1.find("nb=160") != std::string::npos &&
          k1.find("nbeta=320") != std::string::npos);
    pw_tuning t{}, r{};
    CHECK(!read_cache(path, k1, &r));            // no file yet
    CHECK(!read_cache(nullptr, k1, &r));
    CHECK(!read_cache("", k1, &r));
    append_cache("", k1, t);                     // no-op
    t.band_chunk_bytes = 100663296; t.plane_bands = 3; t.z_columns = 64; t.gemm_splits = 29;
    append_cache(path, k1, t);
    CHECK(read_cache(path, k1, &r));
    CHECK(r.band_chunk_bytes == 100663296 && r.plane_bands == 3 && r.z_columns == 64 && r.gemm_splits == 29);
    CHECK(!read_cache(path, k2, &r));
    {   // malformed lines are skipped, the last matching line wins
        FILE *f = std::fopen(path, "a");
        std::fprintf(f, "no tab on this line\n%s\tnot numbers\n%s\t1 2\n", k1.c_str(), k1.c_str());
        std::fclose(f);
    }
    CHECK(read_cache(path, k1, &r) && r.gemm_splits == 29);
    t.gemm_splits = 8; t.plane_bands = 1;
    append_cache(path, k1, t);
    pw_tuning u{}; u.band_chunk_bytes = 1 << 24;
    append_cache(path, k2, u);
    CHECK(read_cache(path, k1, &r) && r.gemm_splits == 8 && r.plane_bands == 1);
    CHECK(read_cache(path, k2, &r) && r.band_chunk_bytes == (1 << 24) && r.gemm_splits == 0);
    for (int i = 0; i < 5; ++i) CHECK(r.reserved[i] == 0);
    // descent: the defaults (t = 1.0) stay unless a candidate beats them by 0.5 %
    std::map<long long, double> ms = {{16, 1.0}, {24, 0.996}, {32, -1.0}, {48, 0.90}, {72, 0.899}, {96, 0.95}};
    pw_tuning best{};
    double tbest = 1.0;
    auto eval = [&](const pw_tuning &c) { return ms.at(c.band_chunk_bytes >> 20); };
    auto set = [](pw_tuning &c, int64_t v) { c.band_chunk_bytes = v << 20; };
    descend(best, tbest, eval, set, {16, 24, 32});
    CHECK(best.band_chunk_bytes == 0 && tbest == 1.0);      // 0.996 is inside the 0.5 % band, 32 failed
    descend(best, tbest, eval, set, {16, 24, 32, 48, 72, 96});
    CHECK(best.band_chunk_bytes == (48ll << 20) && tbest == 0.90);   // 0.899 is not 0.5 % below 0.90
    CHECK(faster(0.5, 1.0) && !faster(0.996, 1.0) && !faster(-1.0, 1.0) && !faster(0.0, 1.0));
    std::printf("%s\n", fails ? "FAILED" : "OK");
    return fails ? 1 : 0;
}
'''


def test_tune_cache_and_descent(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "tune.cpp"
    src.write_text(PROG)
    exe = str(tmp_path / "tune")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", CSRC, str(src), "-o", exe], check=True,
                   capture_output=True)
    r = subprocess.run([exe, str(tmp_path / "cache.txt")], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
