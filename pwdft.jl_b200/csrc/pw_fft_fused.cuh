// Line FFTs with composite radices held entirely in registers.
//
// Same in-place Stockham stages and warp-group organisation as
// pw_fft_tmpl.cuh, but a stage may use a composite radix R = R1*R2 whose
// R-point DFT runs inside one thread (Cooley-Tukey split: R2 DFTs of size R1,
// twiddles W_R^(n2 k1), R1 DFTs of size R2).  Fewer stages means fewer
// shared-memory round trips per line: 75 = 15*5 and 120 = 15*8 take two
// passes instead of three, 27 takes one.
#pragma once
#include "pw_fft.cuh"
#include <type_traits>

namespace pwf {

template <typename T, int R> struct Dft;

// radices with direct formulas
template <typename T> struct Dft<T, 2> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *, int) { SmallDft<T, 2>::run(v, s); } };
template <typename T> struct Dft<T, 3> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *, int) { SmallDft<T, 3>::run(v, s); } };
template <typename T> struct Dft<T, 4> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *, int) { SmallDft<T, 4>::run(v, s); } };
template <typename T> struct Dft<T, 5> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *, int) { SmallDft<T, 5>::run(v, s); } };
template <typename T> struct Dft<T, 8> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *, int) { SmallDft<T, 8>::run(v, s); } };

// exp(-2 pi i m / R) evaluated at compile time: Taylor series of sin and
// cos about 0 after reduction to [-pi, pi] (30 terms: below 1e-17 there).
__host__ __device__ constexpr double ce_trig(double x, bool sine) {
    constexpr double PI = 3.14159265358979323846264338327950288;
    while (x > PI) x -= 2 * PI;
    while (x < -PI) x += 2 * PI;
    double term = sine ? x : 1.0, sum = term;
    for (int k = 1; k < 30; ++k) {
        const int a = sine ? 2 * k : 2 * k - 1, b = sine ? 2 * k + 1 : 2 * k;
        term *= -x * x / ((double)a * (double)b);
        sum += term;
    }
    return sum;
}
template <int M, int R> struct Root {
    static constexpr double ang = -2.0 * 3.14159265358979323846264338327950288 * (double)(M % R) / (double)R;
    static constexpr double c = ce_trig(ang, false), s = ce_trig(ang, true);
};

// compile-time loop: f(std::integral_constant<int, I>) for I in [I0, I1)
template <int I0, int I1, class F> __host__ __device__ __forceinline__ void sfor(F &&f) {
    if constexpr (I0 < I1) {
        f(std::integral_constant<int, I0>{});
        sfor<I0 + 1, I1>(f);
    }
}

// R = R1*R2 in registers, twiddles W_R^(n2 k1) as compile-time constants
// (no table reads; tw and step pass through to the sub-DFTs, which ignore
// them too).
template <typename T, int R1, int R2> struct CompDft {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int step) {
        constexpr int R = R1 * R2;
        Cx<T> a[R];
        sfor<0, R2>([&](auto n2c) {
            constexpr int n2 = decltype(n2c)::value;
            Cx<T> t[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
            Dft<T, R1>::run(t, s, tw, step * R2);
            sfor<0, R1>([&](auto k1c) {
                constexpr int k1 = decltype(k1c)::value;
                if constexpr (n2 * k1 != 0) {
                    using W = Root<n2 * k1, R>;
                    const T wy = s > 0 ? (T)-W::s : (T)W::s;
                    t[k1] = cmul(t[k1], cmake((T)W::c, wy));
                }
                a[n2 * R1 + k1] = t[k1];
            });
        });
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            Cx<T> t[R2];
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[n2 * R1 + k1];
            Dft<T, R2>::run(t, s, tw, step * R1);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
        }
    }
};
// R = R1*R2 with gcd(R1, R2) = 1 (Good-Thomas prime-factor split): input
// n = (R2 n1 + R1 n2) mod R and output k = CRT(k1 mod R1, k2 mod R2) turn
// W_R^(nk) into W_R1^(n1 k1) W_R2^(n2 k2), so no twiddles sit between the
// R2 DFTs of size R1 and the R1 DFTs of size R2 (both index maps are
// compile-time register permutations).
template <int A, int M> __host__ __device__ constexpr int inv_mod() {
    int r = 1;
    while ((A * r) % M != 1) ++r;
    return r;
}
template <typename T, int R1, int R2> struct PfaDft {
    static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int step) {
        constexpr int R = R1 * R2;
        constexpr int E1 = R2 * inv_mod<R2 % R1, R1>(), E2 = R1 * inv_mod<R1 % R2, R2>();   // CRT idempotents
        Cx<T> a[R];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
            Cx<T> t[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[(R2 * n1 + R1 * n2) % R];
            Dft<T, R1>::run(t, s, tw, step);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) a[n2 * R1 + k1] = t[k1];
        }
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            Cx<T> t[R2];
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[n2 * R1 + k1];
            Dft<T, R2>::run(t, s, tw, step);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[(E1 * k1 + E2 * k2) % R] = t[k2];
        }
    }
};
template <typename T> struct Dft<T, 9> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int st) { CompDft<T, 3, 3>::run(v, s, tw, st); } };
template <typename T> struct Dft<T, 15> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int st) { PfaDft<T, 3, 5>::run(v, s, tw, st); } };
template <typename T> struct Dft<T, 24> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int st) { CompDft<T, 8, 3>::run(v, s, tw, st); } };
template <typename T> struct Dft<T, 25> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int st) { CompDft<T, 5, 5>::run(v, s, tw, st); } };
template <typename T> struct Dft<T, 27> { static __host__ __device__ __forceinline__ void run(Cx<T> *v, T s, const Cx<T> *tw, int st) { CompDft<T, 9, 3>::run(v, s, tw, st); } };

// Fused plans: radices per stage (product = N).
template <int N> struct FPlan;
template <> struct FPlan<27> { static constexpr int nst = 1; static __host__ __device__ constexpr int r(int) { return 27; } };
template <> struct FPlan<75> { static constexpr int nst = 2; static __host__ __device__ constexpr int r(int s) { return s == 0 ? 15 : 5; } };
// 120 = 15 * 8: 91-110 registers in the z and plane kernels (24 * 5 needed 128 and spilled
// 72-432 bytes); measured Si216 FFT round trip 7.95 -> 6.52 ms
template <> struct FPlan<120> { static constexpr int nst = 2; static __host__ __device__ constexpr int r(int s) { return s == 0 ? 15 : 8; } };

template <int N> __host__ __device__ constexpr int fp_ns(int s) {
    int p = 1;
    for (int i = 0; i < s; ++i) p *= FPlan<N>::r(i);
    return p;
}
// lines per warp group: the stage with the fewest butterflies per line fills 32 lanes
template <int N> __host__ __device__ constexpr int fp_group() {
    int mn = N;
    for (int s = 0; s < FPlan<N>::nst; ++s) {
        const int nbf = N / FPlan<N>::r(s);
        mn = nbf < mn ? nbf : mn;
    }
    return 32 / mn > 0 ? 32 / mn : 1;
}

// Shared-memory twiddle layout of the fused plans.  One-stage plans keep
// tw[m] = exp(-2 pi i m / N).  Two-stage plans (N = R0 R1) store
//   tw[m]                     = exp(-2 pi i m / R0)   for m < R0 (the
//                               composite DFTs now hold their roots as
//                               compile-time constants and do not read them);
//   tw[R0 + (r - 1) R0 + j]   = exp(-2 pi i r j / N)  for 1 <= r < R1, j < R0,
//                               the stage-1 twiddles, which lanes with
//                               consecutive j read from consecutive words
// (the natural table read at r j puts 2 and 4 lanes of a half-warp on one
// bank for r = 2 and 4).  N entries either way; tw_src(i) is the natural
// index of entry i, for filling the table from tw[m] = exp(-2 pi i m / N).
template <int N> __host__ __device__ constexpr int tw_src(int i) {
    if constexpr (FPlan<N>::nst == 1) {
        return i;
    } else {
        constexpr int R0 = FPlan<N>::r(0);
        return i < R0 ? i * (N / R0) : ((i - R0) / R0 + 1) * ((i - R0) % R0);
    }
}
// step argument of the DFT of stage S: the radix-R0 roots sit at stride 1;
// the stage-1 radix of a two-stage plan reads no table
template <int R> __host__ __device__ constexpr bool direct_radix() { return R == 2 || R == 3 || R == 4 || R == 5 || R == 8; }
template <int N, int S> __host__ __device__ constexpr int tw_step() {
    static_assert(FPlan<N>::nst == 1 || direct_radix<FPlan<N>::r(1)>(), "two-stage plans end on a direct radix");
    return (FPlan<N>::nst == 2 && S == 0) ? 1 : N / FPlan<N>::r(S);
}
// twiddle of element r of stage-S butterfly jm (jm < N_S, the stage's span)
// Padded element positions of a line held in shared memory: pos(x) = x +
// (x / R0) * fp_pad, line stride fp_xs.  A plan whose first-stage outputs put
// several lanes of a half-warp on one bank can pad here (the earlier
// 120 = 24 * 5 plan needed one spare word per 24 elements and stride 125);
// the current plans are unpadded.
template <int N> __host__ __device__ constexpr int fp_pad() { return 0; }
template <int N> __host__ __device__ constexpr int fp_pos(int x) {
    if constexpr (fp_pad<N>() == 0)
        return x;
    else
        return x + (x / FPlan<N>::r(0)) * fp_pad<N>();
}
template <int N> __host__ __device__ constexpr int fp_xs() { return fp_pad<N>() == 0 ? N : N + N / FPlan<N>::r(0) * fp_pad<N>() + 1; }
static_assert(fp_xs<120>() >= fp_pos<120>(119) + 1, "padded line fits its stride");

template <int N, int S> __device__ __forceinline__ int tw_at(int r, int jm) {
    if constexpr (FPlan<N>::nst == 2 && S == 1) {
        constexpr int R0 = FPlan<N>::r(0);
        return R0 + (r - 1) * R0 + jm;
    } else {
        constexpr int R = FPlan<N>::r(S);
        return r * jm * (N / (fp_ns<N>(S) * R));
    }
}

// Lane assignment of round t of a stage with NBF butterflies per line and
// G lines per warp group.  Shared memory serves an 8-byte access one
// half-warp at a time, so with NBF <= 16 every half-warp takes whole lines
// (H = 16 / NBF of them, the rest of its lanes idle): its accesses are then H
// runs of NBF consecutive elements, one per line, instead of runs that
// straddle a line boundary onto banks the half-warp already uses (measured
// model of the 75-point plane kernel: 27 % of its shared-memory wavefronts
// were such conflicts).  The number of rounds equals the packed mapping's
// for every plan here (75: 5 and 15 butterflies, 6 lines; 120: 8 and 15, 4;
// 27: 1, 32).
template <int NBF, int G> struct LaneMap {
    static constexpr int H = NBF <= 16 ? 16 / NBF : 0;
    static constexpr int ROUNDS = H ? (G + 2 * H - 1) / (2 * H) : (G * NBF + 31) / 32;
    static __host__ __device__ __forceinline__ bool at(int lane, int t, int nl, int &line, int &j) {
        if constexpr (H > 0) {
            const int sub = lane & 15, li = sub / NBF;
            j = sub - li * NBF;
            line = (2 * t + (lane >> 4)) * H + li;
            return li < H && line < nl;
        } else {
            const int id = lane + 32 * t;
            line = id / NBF;
            j = id - line * NBF;
            return id < nl * NBF;
        }
    }
};

// w[r] = w1^r for r < R, w[r] = w[r / 2] w[r - r / 2] (about log2(r) + 1
// roundings): the stage twiddles of one butterfly from a single table read.
template <typename T, int R> __device__ __forceinline__ void tw_pow(Cx<T> w1, Cx<T> (&w)[R]) {
    w[0] = cmake((T)1, (T)0);
    if constexpr (R > 1) w[1] = w1;
#pragma unroll
    for (int r = 2; r < R; ++r) w[r] = cmul(w[r / 2], w[r - r / 2]);
}

// Twiddles of butterfly jm of stage S (conjugated for the inverse, sign > 0)
// applied to v[1 .. R).  Only the second stage of a two-stage plan has any;
// its table entry tw_at(1, jm) is exp(-2 pi i jm / N).
template <typename T, int N, int S, int R>
__device__ __forceinline__ void apply_tw(Cx<T> (&v)[R], const Cx<T> *tw, int jm, int sign) {
    Cx<T> w1 = tw[tw_at<N, S>(1, jm)];
    if (sign > 0) w1.y = -w1.y;
    Cx<T> w[R];
    tw_pow<T, R>(w1, w);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
}

// PAD: elements at fp_pos(x) (es must be 1)
template <typename T, int N, int S, bool JFAST, bool PAD>
__device__ __forceinline__ void fstage(Cx<T> *buf, int l0, int nl, int es, int ls, const Cx<T> *tw, int sign, int lane) {
    constexpr int R = FPlan<N>::r(S);
    constexpr int NS = fp_ns<N>(S);
    constexpr int NBF = N / R;
    constexpr int G = fp_group<N>();
    using LM = LaneMap<NBF, G>;
    // JFAST lines: whole lines per half-warp; otherwise (z columns, line
    // index fastest) the packed order, whose strides the callers choose
    constexpr int MAXB = JFAST ? LM::ROUNDS : (G * NBF + 31) / 32;
    auto slot = [&](int t, int &line, int &j) -> bool {
        if constexpr (JFAST) {
            const bool ok = LM::at(lane, t, nl, line, j);
            line += l0;
            return ok;
        } else {
            const int id = lane + 32 * t;
            line = l0 + id % nl;
            j = id / nl;
            return id < nl * NBF;
        }
    };
    const T sg = (T)sign;
    Cx<T> v[MAXB][R];
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        int line, j;
        if (slot(t, line, j)) {
            const int jm = j % NS;
            const Cx<T> *p = buf + line * ls + j * es;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = PAD ? buf[line * ls + fp_pos<N>(j + r * NBF)] : p[r * NBF * es];
            if constexpr (NS > 1) apply_tw<T, N, S, R>(v[t], tw, jm, sign);
            Dft<T, R>::run(v[t], sg, tw, tw_step<N, S>());
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < MAXB; ++t) {
        int line, j;
        if (slot(t, line, j)) {
            const int jm = j % NS;
            const int x0 = (j / NS) * NS * R + jm;
            Cx<T> *q = buf + line * ls + x0 * es;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (PAD)
                    buf[line * ls + fp_pos<N>(x0 + r * NS)] = v[t][r];
                else
                    q[r * NS * es] = v[t][r];
            }
        }
    }
    __syncwarp();
    if constexpr (S + 1 < FPlan<N>::nst) fstage<T, N, S + 1, JFAST, PAD>(buf, l0, nl, es, ls, tw, sign, lane);
}

// All lines [0, nlines) of length N; ends with __syncthreads().
template <typename T, int N, bool JFAST, bool PAD = false>
__device__ __forceinline__ void lines(Cx<T> *buf, int nlines, int es, int ls, const Cx<T> *tw, int sign) {
    constexpr int G = fp_group<N>();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int l0 = warp * G; l0 < nlines; l0 += nw * G) {
        const int nl = min(G, nlines - l0);
        fstage<T, N, 0, JFAST, PAD>(buf, l0, nl, es, ls, tw, sign, lane);
    }
    __syncthreads();
}

}  // namespace pwf

namespace pwf {

// Stage S of the N-point line FFT for lines [0, nl) of one warp group, with
// element access through functors ld(line, x, r) -> Cx<T> and
// st(line, x, r, v) (x the element, r the compile-time slot of the lane's
// butterfly it sits in): the first stage of a line can read its input
// straight from another layout, the last can scale or scatter its output,
// with no extra pass.
template <typename T, int N, int S, class LD, class ST>
__device__ __forceinline__ void fstage_io(int nl, const Cx<T> *tw, int sign, int lane, LD &ld, ST &st) {
    constexpr int R = FPlan<N>::r(S);
    constexpr int NS = fp_ns<N>(S);
    constexpr int NBF = N / R;
    constexpr int G = fp_group<N>();
    using LM = LaneMap<NBF, G>;
    const T sg = (T)sign;
    Cx<T> v[LM::ROUNDS][R];
#pragma unroll
    for (int t = 0; t < LM::ROUNDS; ++t) {
        int line, j;
        if (LM::at(lane, t, nl, line, j)) {
            const int jm = j % NS;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = ld(line, j + r * NBF, r);
            if constexpr (NS > 1) apply_tw<T, N, S, R>(v[t], tw, jm, sign);
            Dft<T, R>::run(v[t], sg, tw, tw_step<N, S>());
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < LM::ROUNDS; ++t) {
        int line, j;
        if (LM::at(lane, t, nl, line, j)) {
            const int jm = j % NS;
            const int x0 = (j / NS) * NS * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) st(line, x0 + r * NS, r, v[t][r]);
        }
    }
    __syncwarp();
}

// Whole N-point FFT of nl <= fp_group<N>() lines held by one warp in buf
// (line stride fp_xs, padded positions): the first stage reads through ld0,
// the last writes through stl, the stages between use buf.
template <typename T, int N, class LD0, class STL>
__device__ __forceinline__ void group_fft(Cx<T> *buf, int nl, const Cx<T> *tw, int sign, int lane, LD0 &ld0, STL &stl) {
    constexpr int XS = fp_xs<N>();
    auto bld = [&](int line, int x, int) { return buf[line * XS + fp_pos<N>(x)]; };
    auto bst = [&](int line, int x, int, Cx<T> v) { buf[line * XS + fp_pos<N>(x)] = v; };
    constexpr int NST = FPlan<N>::nst;
    static_assert(NST == 1 || NST == 2, "fused plans have one or two stages");
    if constexpr (NST == 1) {
        fstage_io<T, N, 0>(nl, tw, sign, lane, ld0, stl);
    } else {
        fstage_io<T, N, 0>(nl, tw, sign, lane, ld0, bst);
        fstage_io<T, N, 1>(nl, tw, sign, lane, bld, stl);
    }
}

// Inverse N-point FFT, pointwise scale, forward FFT of nl <= fp_group<N>()
// lines held by one warp: the op_V_loc x-pass.  The inverse's last stage
// leaves lane (line, j) holding f[j + R0 r], r < R1 (N = R0 R1), which is
// exactly the input of a decimation-in-frequency forward step,
//   F[k2 + R1 k1] = sum_j w_R0^(j k1) [w_N^(j k2) sum_r f[j + R0 r] w_R1^(r k2)],
// so the scale (vsc(line, x)), the forward radix-R1 DFT and its twiddles
// stay in registers and one shared-memory exchange (buf) precedes the
// radix-R0 DFTs, whose outputs go out through st(line, x, r, v).  One-stage
// plans (one line per lane) never touch buf.
template <typename T, int N, class LD0, class VS, class ST>
__device__ __forceinline__ void group_fft_vpair(Cx<T> *buf, int nl, const Cx<T> *tw, int lane, LD0 &ld0, VS &vsc,
                                                ST &st) {
    constexpr int NST = FPlan<N>::nst;
    static_assert(NST == 1 || NST == 2, "fused plans have one or two stages");
    if constexpr (NST == 1) {
        if (lane < nl) {
            Cx<T> v[N];
#pragma unroll
            for (int r = 0; r < N; ++r) v[r] = ld0(lane, r, r);
            Dft<T, N>::run(v, (T)1, tw, 1);
#pragma unroll
            for (int r = 0; r < N; ++r) v[r] = cscale(v[r], vsc(lane, r));
            Dft<T, N>::run(v, (T)-1, tw, 1);
#pragma unroll
            for (int k = 0; k < N; ++k) st(lane, k, k, v[k]);
        }
        __syncwarp();
    } else {
        constexpr int R0 = FPlan<N>::r(0), R1 = FPlan<N>::r(1);
        constexpr int G = fp_group<N>();
        constexpr int XS = fp_xs<N>(), RP = R0 + fp_pad<N>();   // fp_pos(j + R0 r) = j + RP r for j < R0
        auto bst = [&](int line, int x, int, Cx<T> v) { buf[line * XS + fp_pos<N>(x)] = v; };
        fstage_io<T, N, 0>(nl, tw, 1, lane, ld0, bst);   // inverse stage 0 into buf
        using L1 = LaneMap<R0, G>;                         // stage-1 butterflies: R0 per line
        Cx<T> v[L1::ROUNDS][R1];
#pragma unroll
        for (int t = 0; t < L1::ROUNDS; ++t) {
            int line, j;
            if (L1::at(lane, t, nl, line, j)) {
#pragma unroll
                for (int r = 0; r < R1; ++r) v[t][r] = buf[line * XS + j + r * RP];
                apply_tw<T, N, 1, R1>(v[t], tw, j, +1);
                Dft<T, R1>::run(v[t], (T)1, tw, N / R1);      // v[r] = f[j + R0 r]
#pragma unroll
                for (int r = 0; r < R1; ++r) v[t][r] = cscale(v[t][r], vsc(line, j + R0 * r));
                Dft<T, R1>::run(v[t], (T)-1, tw, N / R1);     // sum_r f[j + R0 r] w_R1^(r k2)
                apply_tw<T, N, 1, R1>(v[t], tw, j, -1);
            }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < L1::ROUNDS; ++t) {
            int line, j;
            if (L1::at(lane, t, nl, line, j)) {
#pragma unroll
                for (int k2 = 0; k2 < R1; ++k2) buf[line * XS + k2 * RP + j] = v[t][k2];
            }
        }
        __syncwarp();
        using L2 = LaneMap<R1, G>;                         // radix-R0 butterflies: R1 per line
#pragma unroll
        for (int t = 0; t < L2::ROUNDS; ++t) {
            int line, k2;
            if (L2::at(lane, t, nl, line, k2)) {
                Cx<T> u[R0];
#pragma unroll
                for (int j = 0; j < R0; ++j) u[j] = buf[line * XS + k2 * RP + j];
                Dft<T, R0>::run(u, (T)-1, tw, tw_step<N, 0>());
#pragma unroll
                for (int k1 = 0; k1 < R0; ++k1) st(line, k2 + R1 * k1, k1, u[k1]);
            }
        }
        __syncwarp();
    }
}

}  // namespace pwf
