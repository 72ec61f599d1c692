// Batched 1-D FFTs of short lines held in shared memory.
//
// In-place mixed-radix Stockham autosort (decimation in time): for a stage
// of radix R with Ns = product of the radices already applied, butterfly j
// (0 <= j < n/R) reads x[j + r*n/R], multiplies input r by w_{Ns*R}^{r*(j mod Ns)},
// applies an R-point DFT and writes x[(j/Ns)*Ns*R + (j mod Ns) + r*Ns].
// After the last stage the result is in natural order.  A stage is made
// in-place by having every thread hold its butterflies in registers between
// a read phase and a write phase separated by __syncthreads(); lines are
// processed in whole-line rounds so that no line is read after another
// thread has started writing it.
//
// sign = -1: forward transform (R_to_G, FFTW_FORWARD, exp(-2 pi i/n));
// sign = +1: backward transform, unnormalised (G_to_R times N).
// Twiddles: tw[m] = exp(-2 pi i m / n), computed on the host in FP64.
#pragma once
#include "pw_common.cuh"

// Mathematical constants of the 3-, 5- and 8-point DFTs.
#define PW_SQRT3_2 0.86602540378443864676    // sin(2 pi/3)
#define PW_C5_1    0.30901699437494742410    // cos(2 pi/5) = (sqrt5 - 1)/4
#define PW_C5_2   -0.80901699437494742410    // cos(4 pi/5) = -(sqrt5 + 1)/4
#define PW_S5_1    0.95105651629515357212    // sin(2 pi/5)
#define PW_S5_2    0.58778525229247312917    // sin(4 pi/5)
#define PW_RSQRT2  0.70710678118654752440    // 1/sqrt2

template <typename T, int R> struct SmallDft;

template <typename T> struct SmallDft<T, 2> {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T) {
        Cx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <typename T> struct SmallDft<T, 3> {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s) {
        Cx<T> t1 = cadd(v[1], v[2]);
        Cx<T> t2 = csub(v[0], cscale(t1, (T)0.5));
        Cx<T> t3 = cmul_is(cscale(csub(v[1], v[2]), (T)PW_SQRT3_2), s);
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    }
};

template <typename T> struct SmallDft<T, 4> {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s) {
        Cx<T> a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        Cx<T> c = cadd(v[1], v[3]), d = cmul_is(csub(v[1], v[3]), s);
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        v[1] = cadd(b, d);
        v[3] = csub(b, d);
    }
};

template <typename T> struct SmallDft<T, 5> {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s) {
        Cx<T> a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        Cx<T> a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        Cx<T> x0 = v[0];
        Cx<T> r1 = cadd(x0, cadd(cscale(a1, (T)PW_C5_1), cscale(a2, (T)PW_C5_2)));
        Cx<T> r2 = cadd(x0, cadd(cscale(a1, (T)PW_C5_2), cscale(a2, (T)PW_C5_1)));
        Cx<T> i1 = cmul_is(cadd(cscale(b1, (T)PW_S5_1), cscale(b2, (T)PW_S5_2)), s);
        Cx<T> i2 = cmul_is(csub(cscale(b1, (T)PW_S5_2), cscale(b2, (T)PW_S5_1)), s);
        v[0] = cadd(x0, cadd(a1, a2));
        v[1] = cadd(r1, i1);
        v[4] = csub(r1, i1);
        v[2] = cadd(r2, i2);
        v[3] = csub(r2, i2);
    }
};

template <typename T> struct SmallDft<T, 8> {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s) {
        Cx<T> e[4] = {v[0], v[2], v[4], v[6]};
        Cx<T> o[4] = {v[1], v[3], v[5], v[7]};
        SmallDft<T, 4>::run(e, s);
        SmallDft<T, 4>::run(o, s);
        // w8^k, k = 1..3, w8 = (1 + i s)/sqrt2
        const T h = (T)PW_RSQRT2;
        Cx<T> o1 = cmake(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));
        Cx<T> o2 = cmul_is(o[2], s);
        Cx<T> o3 = cmake(h * (-o[3].x - s * o[3].y), h * (-o[3].y + s * o[3].x));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

// FP32 butterflies on the paired FP32 pipe of sm_100 (one FFMA2 / FADD2 /
// FMUL2 per complex add, real-constant multiply-add or real scale, where
// the scalar formulas above take two).  A product by +-i is folded into
// the FFMA2 that consumes it: r + i s u = (r.x - s u.y, r.y + s u.x) is one
// FFMA2 of the swapped pair (u.y, u.x) with (-s, s); where the operand is
// a difference, the swapped pair is formed directly by two scalar
// subtractions.  Host builds take the same lane-wise formulas with fmaf.
namespace pk {
__host__ __device__ __forceinline__ float2 bc(float c) { return make_float2(c, c); }
__host__ __device__ __forceinline__ float2 add(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 mul(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}
// a * b + c per lane, one rounding
__host__ __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __ffma2_rn(a, b, c);
#else
    return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
// a - b (exact product by -1, one rounding: the same value as a scalar subtraction)
__host__ __device__ __forceinline__ float2 sub(float2 a, float2 b) { return fma(b, bc(-1.0f), a); }
// (a - b) with its lanes swapped: (a.y - b.y, a.x - b.x)
__host__ __device__ __forceinline__ float2 subsw(float2 a, float2 b) { return make_float2(a.y - b.y, a.x - b.x); }
__host__ __device__ __forceinline__ float2 swp(float2 a) { return make_float2(a.y, a.x); }
}  // namespace pk

template <> struct SmallDft<float, 2> {
    static __host__ __device__ __forceinline__ void run(float2 *v, float) {
        const float2 a = v[0], b = v[1];
        v[0] = pk::add(a, b);
        v[1] = pk::sub(a, b);
    }
};

template <> struct SmallDft<float, 3> {
    static __host__ __device__ __forceinline__ void run(float2 *v, float s) {
        const float sc = s * (float)PW_SQRT3_2;
        const float2 t1 = pk::add(v[1], v[2]);
        const float2 t2 = pk::fma(t1, pk::bc(-0.5f), v[0]);
        const float2 ds = pk::subsw(v[1], v[2]);        // i s sqrt3/2 (v1 - v2) = (-sc ds.x, sc ds.y)
        v[0] = pk::add(v[0], t1);
        v[1] = pk::fma(ds, make_float2(-sc, sc), t2);
        v[2] = pk::fma(ds, make_float2(sc, -sc), t2);
    }
};

template <> struct SmallDft<float, 4> {
    static __host__ __device__ __forceinline__ void run(float2 *v, float s) {
        const float2 a = pk::add(v[0], v[2]), b = pk::sub(v[0], v[2]);
        const float2 c = pk::add(v[1], v[3]);
        const float2 ds = pk::subsw(v[1], v[3]);        // i s (v1 - v3) = (-s ds.x, s ds.y)
        v[0] = pk::add(a, c);
        v[2] = pk::sub(a, c);
        v[1] = pk::fma(ds, make_float2(-s, s), b);
        v[3] = pk::fma(ds, make_float2(s, -s), b);
    }
};

template <> struct SmallDft<float, 5> {
    static __host__ __device__ __forceinline__ void run(float2 *v, float s) {
        const float2 x0 = v[0];
        const float2 a1 = pk::add(v[1], v[4]), a2 = pk::add(v[2], v[3]);
        const float2 b1 = pk::subsw(v[1], v[4]), b2 = pk::subsw(v[2], v[3]);   // swapped differences
        const float2 r1 = pk::fma(a2, pk::bc((float)PW_C5_2), pk::fma(a1, pk::bc((float)PW_C5_1), x0));
        const float2 r2 = pk::fma(a2, pk::bc((float)PW_C5_1), pk::fma(a1, pk::bc((float)PW_C5_2), x0));
        // swapped u1 = b1 S1 + b2 S2 and u2 = b1 S2 - b2 S1; r -+ i s u
        const float2 u1 = pk::fma(b2, pk::bc((float)PW_S5_2), pk::mul(b1, pk::bc((float)PW_S5_1)));
        const float2 u2 = pk::fma(b2, pk::bc(-(float)PW_S5_1), pk::mul(b1, pk::bc((float)PW_S5_2)));
        const float2 pm = make_float2(-s, s), mp = make_float2(s, -s);
        v[0] = pk::add(x0, pk::add(a1, a2));
        v[1] = pk::fma(u1, pm, r1);
        v[4] = pk::fma(u1, mp, r1);
        v[2] = pk::fma(u2, pm, r2);
        v[3] = pk::fma(u2, mp, r2);
    }
};

template <> struct SmallDft<float, 8> {
    static __host__ __device__ __forceinline__ void run(float2 *v, float s) {
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        SmallDft<float, 4>::run(e, s);
        SmallDft<float, 4>::run(o, s);
        const float h = (float)PW_RSQRT2;
        const float2 pm = make_float2(-s, s), mp = make_float2(s, -s);
        // w8 o1 = h (o1 + i s o1); w8^3 o3 = -h (o3 - i s o3); w8^2 o2 = i s o2
        const float2 t1 = pk::fma(pk::swp(o[1]), pm, o[1]);
        const float2 q3 = pk::fma(pk::swp(o[3]), mp, o[3]);
        const float2 o2 = pk::swp(o[2]);
        v[0] = pk::add(e[0], o[0]);
        v[4] = pk::sub(e[0], o[0]);
        v[1] = pk::fma(t1, pk::bc(h), e[1]);
        v[5] = pk::fma(t1, pk::bc(-h), e[1]);
        v[2] = pk::fma(o2, pm, e[2]);
        v[6] = pk::fma(o2, mp, e[2]);
        v[3] = pk::fma(q3, pk::bc(-h), e[3]);
        v[7] = pk::fma(q3, pk::bc(h), e[3]);
    }
};

// One radix-R stage over `nlines` lines of length n; element (line, idx)
// lives at buf[line*ls + idx*es].  Threads are mapped line-fastest.
template <typename T, int R, int MAXV>
__device__ __noinline__ void fft_stage(Cx<T> *buf, int n, int Ns, int nlines, int es, int ls,
                                          const Cx<T> *tw, int sign) {
    constexpr int MAXB = (MAXV / R) > 0 ? (MAXV / R) : 1;
    const int nbf = n / R;
    const int nth = blockDim.x;
    int lpr = (nth * MAXB) / nbf;
    if (lpr < 1) lpr = 1;
    if (lpr > nlines) lpr = nlines;
    const int twstride = n / (Ns * R);
    const T s = (T)sign;
    for (int l0 = 0; l0 < nlines; l0 += lpr) {
        const int nl = min(lpr, nlines - l0);
        const int total = nl * nbf;
        Cx<T> v[MAXB][R];
#pragma unroll
        for (int t = 0; t < MAXB; ++t) {
            const int id = threadIdx.x + t * nth;
            if (id < total) {
                const int line = l0 + id % nl;
                const int j = id / nl;
                const int jm = j % Ns;
                const Cx<T> *p = buf + (size_t)line * ls + (size_t)j * es;
#pragma unroll
                for (int r = 0; r < R; ++r) v[t][r] = p[(size_t)r * nbf * es];
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    Cx<T> w = tw[r * jm * twstride];
                    if (sign > 0) w.y = -w.y;
                    v[t][r] = cmul(v[t][r], w);
                }
                SmallDft<T, R>::run(v[t], s);
            }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < MAXB; ++t) {
            const int id = threadIdx.x + t * nth;
            if (id < total) {
                const int line = l0 + id % nl;
                const int j = id / nl;
                const int jm = j % Ns;
                const int idxD = (j / Ns) * Ns * R + jm;
                Cx<T> *q = buf + (size_t)line * ls + (size_t)idxD * es;
#pragma unroll
                for (int r = 0; r < R; ++r) q[(size_t)r * Ns * es] = v[t][r];
            }
        }
        __syncthreads();
    }
}

// Full transform of `nlines` lines.  Ends with a __syncthreads().
template <typename T, int MAXV>
__device__ void fft_lines(Cx<T> *buf, const FftDim &d, int nlines, int es, int ls, const Cx<T> *tw, int sign) {
    int Ns = 1;
    for (int st = 0; st < d.nstage; ++st) {
        const int R = d.radix[st];
        switch (R) {
        case 2: fft_stage<T, 2, MAXV>(buf, d.n, Ns, nlines, es, ls, tw, sign); break;
        case 3: fft_stage<T, 3, MAXV>(buf, d.n, Ns, nlines, es, ls, tw, sign); break;
        case 4: fft_stage<T, 4, MAXV>(buf, d.n, Ns, nlines, es, ls, tw, sign); break;
        case 5: fft_stage<T, 5, MAXV>(buf, d.n, Ns, nlines, es, ls, tw, sign); break;
        default: fft_stage<T, 8, MAXV>(buf, d.n, Ns, nlines, es, ls, tw, sign); break;
        }
        Ns *= R;
    }
}

// ------------------------------------------------------------------------
// Warp-synchronous variant: each warp owns a group of g whole lines and
// runs every stage of them with __syncwarp() only, so warps proceed
// independently (no CTA-wide barrier per stage).  Requires n/R <= 32*MAXB(R)
// for every stage (checked by fft_warp_ok); ends with a __syncthreads().
template <typename T, int R, int MAXV>
__device__ __noinline__ void warp_stage(Cx<T> *buf, int n, int Ns, int l0, int nl, int es, int ls,
                                           const Cx<T> *tw, int sign, int lane, bool jfast) {
    constexpr int MAXB = (MAXV / R) > 0 ? (MAXV / R) : 1;
    const int nbf = n / R;
    const int total = nl * nbf;
    const int twstride = n / (Ns * R);
    const T s = (T)sign;
    Cx<T> v[MAXB][R];
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        const int id = lane + 32 * t;
        if (id < total) {
            const int line = jfast ? l0 + id / nbf : l0 + id % nl;
            const int j = jfast ? id % nbf : id / nl;
            const int jm = j % Ns;
            const Cx<T> *p = buf + (size_t)line * ls + (size_t)j * es;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = p[(size_t)r * nbf * es];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                Cx<T> w = tw[r * jm * twstride];
                if (sign > 0) w.y = -w.y;
                v[t][r] = cmul(v[t][r], w);
            }
            SmallDft<T, R>::run(v[t], s);
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        const int id = lane + 32 * t;
        if (id < total) {
            const int line = jfast ? l0 + id / nbf : l0 + id % nl;
            const int j = jfast ? id % nbf : id / nl;
            const int jm = j % Ns;
            const int idxD = (j / Ns) * Ns * R + jm;
            Cx<T> *q = buf + (size_t)line * ls + (size_t)idxD * es;
#pragma unroll
            for (int r = 0; r < R; ++r) q[(size_t)r * Ns * es] = v[t][r];
        }
    }
    __syncwarp();
}

template <int MAXV>
__host__ __device__ inline int fft_warp_group(const FftDim &d) {
    int g = 1 << 20;
    for (int st = 0; st < d.nstage; ++st) {
        const int R = d.radix[st];
        const int maxb = (MAXV / R) > 0 ? (MAXV / R) : 1;
        const int gg = (32 * maxb) / (d.n / R);
        g = gg < g ? gg : g;
    }
    return g;
}

template <typename T, int MAXV>
__device__ void fft_lines_w(Cx<T> *buf, const FftDim &d, int nlines, int es, int ls, const Cx<T> *tw, int sign) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int g = fft_warp_group<MAXV>(d);
    if (g < 1) g = 1;
    const bool jfast = (es == 1);
    for (int l0 = warp * g; l0 < nlines; l0 += nw * g) {
        const int nl = min(g, nlines - l0);
        int Ns = 1;
        for (int st = 0; st < d.nstage; ++st) {
            const int R = d.radix[st];
            switch (R) {
            case 2: warp_stage<T, 2, MAXV>(buf, d.n, Ns, l0, nl, es, ls, tw, sign, lane, jfast); break;
            case 3: warp_stage<T, 3, MAXV>(buf, d.n, Ns, l0, nl, es, ls, tw, sign, lane, jfast); break;
            case 4: warp_stage<T, 4, MAXV>(buf, d.n, Ns, l0, nl, es, ls, tw, sign, lane, jfast); break;
            case 5: warp_stage<T, 5, MAXV>(buf, d.n, Ns, l0, nl, es, ls, tw, sign, lane, jfast); break;
            default: warp_stage<T, 8, MAXV>(buf, d.n, Ns, l0, nl, es, ls, tw, sign, lane, jfast); break;
            }
            Ns *= R;
        }
    }
    __syncthreads();
}
