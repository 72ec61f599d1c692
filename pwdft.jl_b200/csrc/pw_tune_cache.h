// Host-only pieces of pw_autotune (pw_tune.cu): the cache key, the text
// cache of earlier choices and the acceptance rule of the coordinate
// descent.  No CUDA here, so the same code is compiled into a host program
// by the CPU tests.
//
// Cache file: one line per choice, "<key>\t<band_chunk_bytes> <plane_bands>
// <z_columns> <gemm_splits>\n"; the last line whose key matches wins, lines
// without a tab or without four numbers are skipped.
#pragma once
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pwb200.h"

namespace pwk {
namespace tune {

// The shape a choice applies to: GPU name, grid, plane waves, active
// columns and x planes, bands, dtype, projector count.
inline std::string cache_key(const char *gpu, const int Ns[3], int ngw, int ncol, int nxa, int nb, int dtype,
                             int nbeta) {
    char b[512];
    std::snprintf(b, sizeof(b), "gpu=%s;Ns=%dx%dx%d;Ngw=%d;Ncol=%d;Nxa=%d;nb=%d;dtype=%d;nbeta=%d", gpu, Ns[0], Ns[1],
                  Ns[2], ngw, ncol, nxa, nb, dtype, nbeta);
    return std::string(b);
}

inline bool read_cache(const char *path, const std::string &key, pw_tuning *t) {
    if (!path || !*path) return false;
    FILE *f = std::fopen(path, "r");
    if (!f) return false;
    char line[1024];
    bool hit = false;
    while (std::fgets(line, sizeof(line), f)) {
        char *tab = std::strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        if (key != line) continue;
        long long chunk = 0;
        int bpc = 0, zc = 0, sp = 0;
        if (std::sscanf(tab + 1, "%lld %d %d %d", &chunk, &bpc, &zc, &sp) == 4) {
            std::memset(t, 0, sizeof(*t));
            t->band_chunk_bytes = chunk;
            t->plane_bands = bpc;
            t->z_columns = zc;
            t->gemm_splits = sp;
            hit = true;   // the last matching line wins
        }
    }
    std::fclose(f);
    return hit;
}

inline void append_cache(const char *path, const std::string &key, const pw_tuning &t) {
    if (!path || !*path) return;
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s\t%lld %d %d %d\n", key.c_str(), (long long)t.band_chunk_bytes, t.plane_bands, t.z_columns,
                 t.gemm_splits);
    std::fclose(f);
}

// A candidate replaces the best so far only if it ran (tm > 0) and is at
// least 0.5 % faster: timing noise does not move the choice away from the
// defaults, which are tried first.
inline bool faster(double tm, double tbest) { return tm > 0 && tm < tbest * 0.995; }

// One coordinate of the descent: each value of one field, set on a copy of
// the best parameters so far, timed by eval (negative: the candidate
// failed); the best set and its time are updated in place.
template <class Eval, class Set>
void descend(pw_tuning &best, double &tbest, Eval &&eval, Set &&set, const std::vector<int64_t> &vals) {
    for (int64_t v : vals) {
        pw_tuning cand = best;
        set(cand, v);
        const double tm = eval(cand);
        if (faster(tm, tbest)) {
            tbest = tm;
            best = cand;
        }
    }
}

}  // namespace tune
}  // namespace pwk
