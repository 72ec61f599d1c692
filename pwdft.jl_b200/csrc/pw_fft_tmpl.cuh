// Compile-time specialised warp-synchronous line FFTs.
//
// Same in-place Stockham stages as pw_fft.cuh (fft_lines_w), but the line
// length N, the radix plan and every index derived from them are template
// constants, so butterfly addressing compiles to multiply/shift sequences
// instead of run-time integer division, and all stages unroll.
#pragma once
#include "pw_fft.cuh"

namespace pwt {

// Greedy radix plan (8, 4, 2, then 3, 5), identical to the host's make_plan.
__host__ __device__ constexpr int plan_radix(int n, int s) {
    for (int st = 0;; ++st) {
        const int r = (n % 8 == 0) ? 8 : (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : (n % 5 == 0) ? 5 : 1;
        if (st == s || r == 1) return r;
        n /= r;
    }
}
__host__ __device__ constexpr int plan_len(int n) {
    int c = 0;
    while (n > 1) {
        const int r = plan_radix(n, 0);
        if (r == 1) return -1;
        n /= r;
        ++c;
    }
    return c;
}
__host__ __device__ constexpr int plan_ns(int n, int s) {
    int p = 1;
    for (int i = 0; i < s; ++i) p *= plan_radix(n, i);
    return p;
}
__host__ __device__ constexpr int maxb_of(int maxv, int r) { return (maxv / r) > 0 ? (maxv / r) : 1; }
// lines per warp group: every stage of a group must fit 32 lanes x MAXB butterflies
__host__ __device__ constexpr int group_lines(int n, int maxv) {
    int g = 1 << 20;
    for (int s = 0; s < plan_len(n); ++s) {
        const int r = plan_radix(n, s);
        const int gg = (32 * maxb_of(maxv, r)) / (n / r);
        g = gg < g ? gg : g;
    }
    return g;
}

template <typename T, int N, int S, int MAXV, bool JFAST>
__device__ __forceinline__ void stage(Cx<T> *buf, int l0, int nl, int es, int ls, const Cx<T> *tw, int sign, int lane) {
    constexpr int R = plan_radix(N, S);
    constexpr int NS = plan_ns(N, S);
    constexpr int NBF = N / R;
    constexpr int MAXB = maxb_of(MAXV, R);
    constexpr int TWS = N / (NS * R);
    const int total = nl * NBF;
    const T sg = (T)sign;
    Cx<T> v[MAXB][R];
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        const int id = lane + 32 * t;
        if (id < total) {
            const int line = JFAST ? l0 + id / NBF : l0 + id % nl;
            const int j = JFAST ? id % NBF : id / nl;
            const int jm = j % NS;
            const Cx<T> *p = buf + line * ls + j * es;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = p[r * NBF * es];
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    Cx<T> w = tw[r * jm * TWS];
                    if (sign > 0) w.y = -w.y;
                    v[t][r] = cmul(v[t][r], w);
                }
            }
            SmallDft<T, R>::run(v[t], sg);
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        const int id = lane + 32 * t;
        if (id < total) {
            const int line = JFAST ? l0 + id / NBF : l0 + id % nl;
            const int j = JFAST ? id % NBF : id / nl;
            const int jm = j % NS;
            Cx<T> *q = buf + line * ls + ((j / NS) * NS * R + jm) * es;
#pragma unroll
            for (int r = 0; r < R; ++r) q[r * NS * es] = v[t][r];
        }
    }
    __syncwarp();
    if constexpr (S + 1 < plan_len(N)) stage<T, N, S + 1, MAXV, JFAST>(buf, l0, nl, es, ls, tw, sign, lane);
}

// All lines [0, nlines) of length N, one warp group of G lines at a time per
// warp.  Ends with __syncthreads().
template <typename T, int N, int MAXV, bool JFAST>
__device__ __forceinline__ void lines(Cx<T> *buf, int nlines, int es, int ls, const Cx<T> *tw, int sign) {
    constexpr int G = group_lines(N, MAXV);
    static_assert(plan_len(N) > 0 && G >= 1, "unsupported line length");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int l0 = warp * G; l0 < nlines; l0 += nw * G) {
        const int nl = min(G, nlines - l0);
        stage<T, N, 0, MAXV, JFAST>(buf, l0, nl, es, ls, tw, sign, lane);
    }
    __syncthreads();
}

}  // namespace pwt
