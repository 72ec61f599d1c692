// Complex GEMMs of the mixed-precision path on the 5th-generation tensor
// cores (tcgen05.mma, kind::f16 with BF16 operands, FP32 accumulation in
// TMEM, operands staged by TMA into 128B-swizzled shared memory).
//
// Every product is brought to one form, C (m x n complex) = Z^H W with
// Z (K x m) and W (K x n):
//   betaNL' psi        (PsPotNL.jl:252)              Z = betaNL,  W = psi
//   X'HX, Q'HQ, Q'Q    (diag_LOBPCG.jl:85,183-184)   Z = Q,       W = HQ / Q
//   A*U                (diag_LOBPCG.jl:188-194,
//                       op_V_Ps_nloc.jl:59-76)       Z = A^H,     W = U
// and embedded as one real GEMM  D (2m x n) = A' B'^T  over K' = 2K with
//   A' row 2i   = [Re z_i, Im z_i] interleaved along K   (z_i = column i of Z)
//   A' row 2i+1 = [-Im z_i, Re z_i]                       (= i z_i)
//   B' row j    = [Re w_j, Im w_j]
// so that D[2i, j] = Re C(i, j) and D[2i+1, j] = Im C(i, j): D stored column-
// major IS the interleaved complex C.
//
// Precision: split BF16 x 3.  Each FP32 operand x = hi + lo with
// hi = bf16(x), lo = bf16(x - hi); A'B'^T ~ hi*hi + hi*lo + lo*hi, all three
// accumulated in the same FP32 TMEM accumulator (relative error ~2^-17 per
// product, then FP32 accumulation).  The "prep" kernels below write the
// K-major BF16 hi/lo operands (transposing where Z = A^H) so that the MMA
// kernel only ever sees K-major A and B.
//
// MMA kernel: 128 x 128 output tile per CTA, BK = 64 (one 128-byte swizzle
// row of BF16), 3-stage TMA -> MMA pipeline on mbarriers, split-K over
// gridDim.z into an FP32 workspace, then a finalize kernel that sums the
// splits and writes the complex result (FP32 or FP64, overwrite or add).
// Warp roles: warp 0 = TMA producer, warp 1 = TMEM owner + MMA issuer,
// warps 2..5 = epilogue (TMEM -> registers -> global).  Every mbarrier wait
// is bounded; on expiry the CTA records an error code and returns after
// releasing its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "pw_launch.h"
#include "pw_umma.h"

namespace pwk {
namespace umma {

constexpr int BM = 128, BK = 64;
constexpr int TILE_A_BYTES = BM * BK * 2;   // 16 KB per A operand tile
constexpr int THREADS = 192;
constexpr long long WAIT_LIMIT = 1ll << 26;
constexpr int MAX_STAGES = 3;
// k-blocks accumulated in one TMEM tile before the epilogue drains it (each
// tile is one accumulation chain of the tensor core's truncating FP32 adds;
// measured: 2 to 8 k-blocks per chain gain at most 6 % on the Si216 Gram and
// bias its diagonal by -6e-7 to -3e-6, one k-block by -1e-7)
#ifndef PW_UMMA_CHAIN
#define PW_UMMA_CHAIN 1
#endif
constexpr int CHAIN = PW_UMMA_CHAIN;

// NS = number of BF16 pieces per FP32 value: 2 (hi, lo: 3 products, ~2^-17)
// or 3 (hi, mid, lo: 6 products, ~2^-24, for products with heavy
// cancellation such as betaNL' psi).  BN = output tile width (complex
// columns): 128, or 160 when it pads n less (n = 160, 480, 1440 bands: one
// MMA of N = 160 instead of two of N = 128 with 96 columns of padding, and
// the A tiles read once per 160 columns).  Stages: as many as fit in 227 KB.
template <int NS, int BN> struct Cfg {
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "tcgen05 N for M = 128, whole 32-column TMEM loads");
    static constexpr int TILE_B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = NS * (TILE_A_BYTES + TILE_B_BYTES);
    static constexpr int STAGES = (225 * 1024) / STAGE_BYTES < MAX_STAGES ? (225 * 1024) / STAGE_BYTES : MAX_STAGES;
    static_assert(STAGES >= 2, "at least a double-buffered pipeline");
    // two accumulator tiles (double buffer), allocation a power of two >= 32
    static constexpr uint32_t TMEM_COLS = 2 * BN <= 256 ? 256u : 512u;
    // kind::f16, A = B = BF16, D = F32, both K-major, M = 128, N = BN
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};

struct __align__(8) Bars {
    uint64_t full[MAX_STAGES];
    uint64_t empty[MAX_STAGES];
    uint64_t tfull[2];    // accumulator tile b holds a finished k-block
    uint64_t tempty[2];   // the epilogue has drained accumulator tile b
    uint32_t tmem_base;
    int failed;
};
template <int NS, int BN> constexpr size_t smem_bytes() {
    return 1024 + (size_t)Cfg<NS, BN>::STAGES * Cfg<NS, BN>::STAGE_BYTES + sizeof(Bars);
}

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity) {
    for (long long i = 0; i < WAIT_LIMIT; ++i)
        if (mbar_try(b, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            su32(dst)),
        "l"((uint64_t)map), "r"(su32(bar)), "r"(c0), "r"(c1)
        : "memory");
}
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
    // K-major, 128B swizzle: LBO = 16 B (unused), SBO = 1024 B (8 rows x 128 B), version 1
    return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// D (Mp x Np) = sum over the split's k-blocks of the piece products
//   NS = 2:  A0 B0^T + A0 B1^T + A1 B0^T
//   NS = 3:  A0 B0^T + A0 B1^T + A1 B0^T + A0 B2^T + A1 B1^T + A2 B0^T
// written to W[z][n][m] (fp32, column-major, ld = Mp), or, with a single
// split (gridDim.z == 1) and C given, straight into the complex result C
// (element (i, j) at C[j ldc + i], rows 2i and 2i + 1 of D its real and
// imaginary parts; cdouble: C is complex128; accumulate: C += D; upper: only
// i <= j written).
template <int NS, int BN>
__global__ void __launch_bounds__(THREADS, 1)
k_umma_gemm(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
            const __grid_constant__ CUtensorMap tA2, const __grid_constant__ CUtensorMap tB0,
            const __grid_constant__ CUtensorMap tB1, const __grid_constant__ CUtensorMap tB2, int Mp, int Np, int KB,
            int kb_per, float *__restrict__ W, int *__restrict__ err, int upper, int lolo, void *__restrict__ C,
            int64_t ldc, int cdouble, int accumulate) {
    using CF = Cfg<NS, BN>;
    constexpr int STAGES = CF::STAGES;
    constexpr int STAGE_BYTES = CF::STAGE_BYTES;
    constexpr int TB = CF::TILE_B_BYTES;
    constexpr int TA = TILE_A_BYTES;
    // upper: C = Z^H W is Hermitian and only its upper triangle is read; a
    // tile whose complex rows (m0/2 ..) all lie below its columns is skipped
    // before any barrier or TMEM allocation
    if (upper && (int)(blockIdx.x * BM) / 2 > (int)(blockIdx.y * BN) + BN - 1) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    Bars *bars = reinterpret_cast<Bars *>(smem + (size_t)STAGES * STAGE_BYTES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int kb0 = blockIdx.z * kb_per;
    const int kb1 = min(KB, kb0 + kb_per);
    const int nkb = max(0, kb1 - kb0);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&bars->full[s], 1);
            mbar_init(&bars->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&bars->tfull[b], 1);
            mbar_init(&bars->tempty[b], 4);   // one arrival per epilogue warp
        }
        bars->failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&bars->tmem_base)),
                     "r"(CF::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = bars->tmem_base;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        for (int i = 0; i < nkb; ++i) {
            const int s = i % STAGES;
            const uint32_t ph = (uint32_t)((i / STAGES) & 1);
            if (!mbar_wait(&bars->empty[s], ph ^ 1)) {
                bars->failed = 1;
                break;
            }
            unsigned char *st = smem + (size_t)s * STAGE_BYTES;
            mbar_expect_tx(&bars->full[s], STAGE_BYTES);
            const int kc = (kb0 + i) * BK;
            // stage layout: A pieces 0..NS-1, then B pieces 0..NS-1
            tma_load_2d(st, &tA0, &bars->full[s], kc, m0);
            tma_load_2d(st + TA, &tA1, &bars->full[s], kc, m0);
            if constexpr (NS == 3) tma_load_2d(st + 2 * TA, &tA2, &bars->full[s], kc, m0);
            tma_load_2d(st + NS * TA, &tB0, &bars->full[s], kc, n0);
            tma_load_2d(st + NS * TA + TB, &tB1, &bars->full[s], kc, n0);
            if constexpr (NS == 3) tma_load_2d(st + NS * TA + 2 * TB, &tB2, &bars->full[s], kc, n0);
        }
        // wait (bounded) for the loads still in flight before leaving
        for (int i = max(0, nkb - STAGES); i < nkb; ++i) {
            const int s = i % STAGES;
            if (!mbar_wait(&bars->full[s], (uint32_t)((i / STAGES) & 1))) bars->failed = 1;
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: every CHAIN k-blocks accumulate into a
        // fresh TMEM tile (b = chain & 1), within a k-block the correction
        // products first and the main product last, so that the tensor
        // core's truncating FP32 accumulation touches each value only a few
        // times; the epilogue sums the tiles with round-to-nearest adds
        for (int i = 0; i < nkb; ++i) {
            const int s = i % STAGES;
            const uint32_t ph = (uint32_t)((i / STAGES) & 1);
            const int ch = i / CHAIN;
            const bool first = i % CHAIN == 0;
            const int b = ch & 1;
            const uint32_t tu = (uint32_t)((ch >> 1) & 1);
            if ((first && !mbar_wait(&bars->tempty[b], tu ^ 1)) || !mbar_wait(&bars->full[s], ph)) {
                bars->failed = 1;
                break;
            }
            fence_after();
            const uint32_t base = su32(smem + (size_t)s * STAGE_BYTES);
            const uint32_t d = tmem + (uint32_t)(b * BN);
            constexpr uint32_t ID = CF::IDESC;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint32_t off = kk * 32;
                const uint64_t a0 = sdesc(base + off), a1 = sdesc(base + TA + off);
                const uint64_t b0 = sdesc(base + NS * TA + off), b1 = sdesc(base + NS * TA + TB + off);
                const bool fresh = first && kk == 0;
                // lolo (two pieces, A and B the same block): the lo*lo term
                // too, whose omission would bias every |z|^2 on the diagonal low
                if (NS == 2 && lolo) mma_bf16(d, a1, b1, ID, fresh ? 0u : 1u);
                mma_bf16(d, a0, b1, ID, (!fresh || (NS == 2 && lolo)) ? 1u : 0u);
                mma_bf16(d, a1, b0, ID, 1u);
                if constexpr (NS == 3) {
                    const uint64_t a2 = sdesc(base + 2 * TA + off), b2 = sdesc(base + NS * TA + 2 * TB + off);
                    mma_bf16(d, a0, b2, ID, 1u);
                    mma_bf16(d, a1, b1, ID, 1u);
                    mma_bf16(d, a2, b0, ID, 1u);
                }
            }
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint32_t off = kk * 32;
                mma_bf16(d, sdesc(base + off), sdesc(base + NS * TA + off), ID, 1u);
            }
            mma_commit(&bars->empty[s]);
            if (i % CHAIN == CHAIN - 1 || i == nkb - 1) mma_commit(&bars->tfull[b]);
        }
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM lanes [32q, 32q+32) -> rows m0 + 32q + lane,
        // the chain tiles summed in registers
        const int q = warp & 3;
        const int m = m0 + 32 * q + lane;
        float acc[BN];
#pragma unroll
        for (int t = 0; t < BN; ++t) acc[t] = 0.f;
        bool ok = true;
        const int nch = (nkb + CHAIN - 1) / CHAIN;
        for (int i = 0; i < nch; ++i) {
            const int b = i & 1;
            const uint32_t tu = (uint32_t)((i >> 1) & 1);
            if (!mbar_wait(&bars->tfull[b], tu)) {
                ok = false;
                break;
            }
            fence_after();
#pragma unroll
            for (int c = 0; c < BN / 32; ++c) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * BN + 32 * c), v);
#pragma unroll
                for (int t = 0; t < 32; ++t) acc[32 * c + t] += v[t];
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars->tempty[b]);
        }
        if (!ok) atomicExch(err, 2);
        if (m < Mp) {
            if (gridDim.z == 1 && C) {
                // lanes hold consecutive rows of D = alternating Re / Im of
                // consecutive complex rows: coalesced component stores
                const int i = m >> 1, part = m & 1;
                if (cdouble) {
                    double *Cd = (double *)C;
#pragma unroll
                    for (int t = 0; t < BN; ++t) {
                        const int n = n0 + t;
                        if (n < Np && !(upper && i > n)) {
                            double *p = Cd + 2 * ((size_t)n * ldc + i) + part;
                            *p = accumulate ? *p + (double)acc[t] : (double)acc[t];
                        }
                    }
                } else {
                    float *Cf = (float *)C;
#pragma unroll
                    for (int t = 0; t < BN; ++t) {
                        const int n = n0 + t;
                        if (n < Np && !(upper && i > n)) {
                            float *p = Cf + 2 * ((size_t)n * ldc + i) + part;
                            *p = accumulate ? *p + acc[t] : acc[t];
                        }
                    }
                }
            } else {
                float *Wz = W + (size_t)blockIdx.z * Mp * (size_t)Np;
#pragma unroll
                for (int t = 0; t < BN; ++t) {
                    const int n = n0 + t;
                    if (n < Np) Wz[(size_t)n * Mp + m] = acc[t];
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && bars->failed) atomicExch(err, 1);
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CF::TMEM_COLS));
    }
}

// ------------------------------------------------------------ prep kernels
__device__ __forceinline__ void split2(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
// x = p[0] + p[1] (+ p[2]): successive BF16 roundings of the remainder
template <int NS> __device__ __forceinline__ void splitn(float x, __nv_bfloat16 *p) {
    p[0] = __float2bfloat16_rn(x);
    const float r = x - __bfloat162float(p[0]);
    p[1] = __float2bfloat16_rn(r);
    if constexpr (NS == 3) p[2] = __float2bfloat16_rn(r - __bfloat162float(p[1]));
}

// A' from Z (K x m, complex, column-major, ld): rows 2i, 2i+1 of length Kp,
// one array per BF16 piece (pc[0..NS-1]).
template <typename CT, int NS>
__global__ void k_prep_tn_a(const CT *__restrict__ Z, int64_t ld, int64_t K, int m, int Kp, __nv_bfloat16 *__restrict__ p0,
                            __nv_bfloat16 *__restrict__ p1, __nv_bfloat16 *__restrict__ p2) {
    const int i = blockIdx.y;
    const CT *z = Z + (size_t)i * ld;
    __nv_bfloat16 *pc[3] = {p0, p1, p2};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < Kp / 2; k += (int64_t)gridDim.x * blockDim.x) {
        float re = 0.f, im = 0.f;
        if (k < K) {
            re = (float)z[k].x;
            im = (float)z[k].y;
        }
        __nv_bfloat16 a[3], c[3];
        splitn<NS>(re, a);
        splitn<NS>(im, c);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            __nv_bfloat16 *r0 = pc[q] + (size_t)(2 * i) * Kp, *r1 = r0 + Kp;
            r0[2 * k] = a[q];
            r0[2 * k + 1] = c[q];
            r1[2 * k] = __hneg(c[q]);  // i z = (-im, re)
            r1[2 * k + 1] = a[q];
        }
    }
}

// B' from W (K x n, complex, column-major, ld): row j = [Re w_j, Im w_j].
template <typename CT, int NS>
__global__ void k_prep_tn_b(const CT *__restrict__ Wm, int64_t ld, int64_t K, int n, int Kp, __nv_bfloat16 *__restrict__ p0,
                            __nv_bfloat16 *__restrict__ p1, __nv_bfloat16 *__restrict__ p2) {
    const int j = blockIdx.y;
    const CT *w = Wm + (size_t)j * ld;
    __nv_bfloat16 *pc[3] = {p0, p1, p2};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < Kp / 2; k += (int64_t)gridDim.x * blockDim.x) {
        float re = 0.f, im = 0.f;
        if (k < K) {
            re = (float)w[k].x;
            im = (float)w[k].y;
        }
        __nv_bfloat16 a[3], c[3];
        splitn<NS>(re, a);
        splitn<NS>(im, c);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            __nv_bfloat16 *r = pc[q] + (size_t)j * Kp;
            r[2 * k] = a[q];
            r[2 * k + 1] = c[q];
        }
    }
}

// A' for Z = A^H, A (M x k complex, column-major, lda): row 2g = [Re, Im] of
// conj(A[g, :]) = [Ar, -Ai]; row 2g+1 = i conj(A[g, :]) = [Ai, Ar].  The
// 32 x 32 tile is transposed through shared memory so both the read of A
// (along g) and the write of A' (along l) are coalesced.
template <typename CT>
__global__ void k_prep_nn_a(const CT *__restrict__ A, int64_t lda, int64_t M, int k, int Kp, __nv_bfloat16 *__restrict__ hi,
                            __nv_bfloat16 *__restrict__ lo) {
    __shared__ float2 tile[32][33];
    const int64_t g0 = (int64_t)blockIdx.x * 32;
    const int l0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int l = l0 + r;
        const int64_t g = g0 + tx;
        float2 v = make_float2(0.f, 0.f);
        if (l < k && g < M) v = make_float2((float)A[(size_t)l * lda + g].x, (float)A[(size_t)l * lda + g].y);
        tile[r][tx] = v;  // tile[l][g]
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int64_t g = g0 + r;
        const int l = l0 + tx;
        if (g >= M || 2 * l >= Kp) continue;
        const float2 v = tile[tx][r];
        __nv_bfloat16 a, b, c, d;
        split2(v.x, a, b);
        split2(v.y, c, d);
        __nv_bfloat16 *h0 = hi + (size_t)(2 * g) * Kp, *h1 = h0 + Kp;
        __nv_bfloat16 *q0 = lo + (size_t)(2 * g) * Kp, *q1 = q0 + Kp;
        h0[2 * l] = a; q0[2 * l] = b;                 // Re conj = Ar
        h0[2 * l + 1] = __hneg(c); q0[2 * l + 1] = __hneg(d);   // Im conj = -Ai
        h1[2 * l] = c; q1[2 * l] = d;                 // Re(i conj) = Ai
        h1[2 * l + 1] = a; q1[2 * l + 1] = b;         // Im(i conj) = Ar
    }
}

// zero the K padding columns [2k, Kp) of every row written by k_prep_nn_a
__global__ void k_zero_pad(__nv_bfloat16 *hi, __nv_bfloat16 *lo, int64_t rows, int Kp, int kfrom) {
    const int w = Kp - kfrom;
    const size_t total = (size_t)rows * w;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / w, c = kfrom + t % w;
        hi[r * Kp + c] = __float2bfloat16_rn(0.f);
        lo[r * Kp + c] = __float2bfloat16_rn(0.f);
    }
}

// C (m x n complex, ldc) (+)= sum_z W[z]  with W[z][j][2i + {0,1}] = {Re, Im}
template <typename CT>
__global__ void k_finalize(const float *__restrict__ W, int S, int m, int n, CT *__restrict__ C, int64_t ldc, int accumulate,
                           int upper) {
    const size_t total = (size_t)m * n;
    const size_t Mp = 2 * (size_t)m;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t j = t / m, i = t - j * m;
        if (upper && i > j) continue;
        double re = 0.0, im = 0.0;
        for (int z = 0; z < S; ++z) {
            const float *w = W + (size_t)z * Mp * n + j * Mp + 2 * i;
            re += (double)w[0];
            im += (double)w[1];
        }
        CT *p = C + j * ldc + i;
        if (accumulate) {
            re += (double)p->x;
            im += (double)p->y;
        }
        p->x = re;
        p->y = im;
    }
}

// ------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

cudaError_t get_encoder() {
    if (g_encode) return cudaSuccess;
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return cudaSuccess;
}

// rows of Kp BF16 values, row r at base + r * rstride * Kp
cudaError_t make_map(CUtensorMap *map, const void *base, int64_t rows, int Kp, int box_rows, int rstride) {
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)Kp * 2 * (cuuint64_t)rstride};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int blocks_for(size_t total) {
    size_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return b < 1 ? 1 : (int)b;
}

}  // namespace umma

using namespace umma;

int umma_kpad(int64_t K) { return (int)(((2 * K + BK - 1) / BK) * BK); }

size_t umma_operand_bytes(int64_t rows, int64_t K) { return (size_t)rows * umma_kpad(K) * 2 * 2; }

template <typename CT>
cudaError_t umma_prep_tn_a(const void *Z, int64_t ld, int64_t K, int m, UmmaOperand &op, cudaStream_t st) {
    op.rows = 2 * (int64_t)m;
    op.Kp = umma_kpad(K);
    dim3 grid((unsigned)std::min<int64_t>((op.Kp / 2 + 255) / 256, 64), m);
    if (op.lo2)
        k_prep_tn_a<CT, 3><<<grid, 256, 0, st>>>((const CT *)Z, ld, K, m, op.Kp, op.hi, op.lo, op.lo2);
    else
        k_prep_tn_a<CT, 2><<<grid, 256, 0, st>>>((const CT *)Z, ld, K, m, op.Kp, op.hi, op.lo, nullptr);
    return cudaGetLastError();
}

template <typename CT>
cudaError_t umma_prep_tn_b(const void *Wm, int64_t ld, int64_t K, int n, UmmaOperand &op, cudaStream_t st) {
    op.rows = n;
    op.Kp = umma_kpad(K);
    dim3 grid((unsigned)std::min<int64_t>((op.Kp / 2 + 255) / 256, 64), n);
    if (op.lo2)
        k_prep_tn_b<CT, 3><<<grid, 256, 0, st>>>((const CT *)Wm, ld, K, n, op.Kp, op.hi, op.lo, op.lo2);
    else
        k_prep_tn_b<CT, 2><<<grid, 256, 0, st>>>((const CT *)Wm, ld, K, n, op.Kp, op.hi, op.lo, nullptr);
    return cudaGetLastError();
}

template <typename CT>
cudaError_t umma_prep_nn_a(const void *A, int64_t lda, int64_t M, int k, UmmaOperand &op, cudaStream_t st) {
    op.rows = 2 * M;
    op.Kp = umma_kpad(k);
    dim3 grid((unsigned)((M + 31) / 32), (k + 31) / 32);
    k_prep_nn_a<CT><<<grid, 256, 0, st>>>((const CT *)A, lda, M, k, op.Kp, op.hi, op.lo);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (op.Kp > 2 * k) {
        k_zero_pad<<<blocks_for((size_t)op.rows * (op.Kp - 2 * k)), 256, 0, st>>>(op.hi, op.lo, op.rows, op.Kp, 2 * k);
        e = cudaGetLastError();
    }
    return e;
}

// Output tile width for n complex columns: 160 when it pads n less than 128
// does (n = 160, 320, 480, 1440), else 128.
static int pick_bn(int n) {
    const int p128 = (n + 127) / 128 * 128, p160 = (n + 159) / 160 * 160;
    return p160 < p128 ? 160 : 128;
}

// Split-K count.  One CTA fits on an SM (222 KB of shared memory); the
// count minimises a model of the run time in k-block units: waves of the
// active tiles (those on or above the diagonal for a Hermitian product) x
// splits over 148 SMs, times the k-blocks per split plus ~8 for a CTA's
// pipeline fill and epilogue, plus the split-K workspace pass.  (Measured:
// the Si64 betaNL' psi at 5 tiles x 60 splits ran as 2 waves plus 4 CTAs;
// the Si216 Gram, 115 active tiles, was slower unsplit than at 2 splits.)
// Accuracy does not depend on it: every CHAIN k-blocks are their own
// accumulation chain in TMEM.
int umma_splits(int64_t Mp, int Np, int Kp, int splits, int upper) {
    const int KB = Kp / BK;
    if (splits > 0) return std::max(1, std::min(splits, KB));
    const int bn = pick_bn(Np);
    const int mt = (int)((Mp + BM - 1) / BM), nt = (Np + bn - 1) / bn;
    int active = mt * nt;
    if (upper) {
        active = 0;
        for (int by = 0; by < nt; ++by)
            for (int bx = 0; bx < mt; ++bx) active += (bx * BM) / 2 > by * bn + bn - 1 ? 0 : 1;
    }
    active = std::max(1, active);
    const int smax = std::max(1, std::min(64, KB / 4));
    int best = 1;
    double tbest = 1e300;
    for (int S = 1; S <= smax; ++S) {
        const double waves = (double)((active * S + 147) / 148);
        const double t = waves * ((double)(KB + S - 1) / S + 8.0) + (S > 1 ? (double)S * Mp * Np / 1.6e6 : 0.0);
        if (t < tbest * (1.0 - 1e-9)) {
            tbest = t;
            best = S;
        }
    }
    return best;
}

size_t umma_ws_bytes(int64_t Mp, int Np, int Kp, int splits, int upper) {
    return (size_t)umma_splits(Mp, Np, Kp, splits, upper) * Mp * Np * sizeof(float);
}

template <int NS, int BN>
static cudaError_t launch_umma(const CUtensorMap *mA, const CUtensorMap *mB, dim3 grid, int Mp, int n, int KB, int kb_per,
                               float *ws, int *err, int upper, int lolo, void *C, int64_t ldc, int cdouble, int accumulate,
                               cudaStream_t st) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_umma_gemm<NS, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_bytes<NS, BN>());
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k_umma_gemm<NS, BN><<<grid, THREADS, smem_bytes<NS, BN>(), st>>>(mA[0], mA[1], mA[2], mB[0], mB[1], mB[2], Mp, n, KB,
                                                                      kb_per, ws, err, upper, lolo, C, ldc, cdouble,
                                                                      accumulate);
    return cudaGetLastError();
}

template <typename CT>
cudaError_t umma_gemm(const UmmaOperand &A, const UmmaOperand &B, int m, int n, void *C, int64_t ldc, int accumulate,
                      float *ws, int *err, cudaStream_t st, int upper, int lolo, int splits) {
    cudaError_t e = get_encoder();
    if (e != cudaSuccess) return e;
    if (A.Kp != B.Kp || A.rows != 2 * (int64_t)m || B.rows != n) return cudaErrorInvalidValue;
    // three BF16 pieces only when both operands carry them
    const int ns = (A.lo2 && B.lo2) ? 3 : 2;
    const int bn = pick_bn(n);
    CUtensorMap mA[3], mB[3];
    const __nv_bfloat16 *pa[3] = {A.hi, A.lo, ns == 3 ? A.lo2 : A.lo};
    const __nv_bfloat16 *pb[3] = {B.hi, B.lo, ns == 3 ? B.lo2 : B.lo};
    for (int q = 0; q < 3; ++q) {
        if ((e = make_map(&mA[q], pa[q], A.rows, A.Kp, BM, A.rstride)) != cudaSuccess) return e;
        if ((e = make_map(&mB[q], pb[q], B.rows, B.Kp, bn, B.rstride)) != cudaSuccess) return e;
    }
    const int KB = A.Kp / BK;
    const int S = umma_splits(A.rows, n, A.Kp, splits, upper);
    const int kb_per = (KB + S - 1) / S;
    dim3 grid((unsigned)((A.rows + BM - 1) / BM), (n + bn - 1) / bn, S);
    // one split and no accumulation: the epilogue writes C itself, no
    // workspace pass (accumulating, its read-modify-write of C measured
    // slower than the workspace + finalize pass: Si64 op_H 0.78 -> 0.95 ms)
    void *Cd = (S == 1 && !accumulate) ? C : nullptr;
    const int cd = sizeof(CT) == 16 ? 1 : 0;
    if (ns == 3)
        e = bn == 160 ? launch_umma<3, 160>(mA, mB, grid, (int)A.rows, n, KB, kb_per, ws, err, upper, 0, Cd, ldc, cd, accumulate, st)
                      : launch_umma<3, 128>(mA, mB, grid, (int)A.rows, n, KB, kb_per, ws, err, upper, 0, Cd, ldc, cd, accumulate, st);
    else
        e = bn == 160 ? launch_umma<2, 160>(mA, mB, grid, (int)A.rows, n, KB, kb_per, ws, err, upper, lolo, Cd, ldc, cd, accumulate, st)
                      : launch_umma<2, 128>(mA, mB, grid, (int)A.rows, n, KB, kb_per, ws, err, upper, lolo, Cd, ldc, cd, accumulate, st);
    if (e != cudaSuccess || Cd) return e;
    k_finalize<CT><<<blocks_for((size_t)m * n), 256, 0, st>>>(ws, S, m, n, (CT *)C, ldc, accumulate, upper);
    return cudaGetLastError();
}

template cudaError_t umma_prep_tn_a<float2>(const void *, int64_t, int64_t, int, UmmaOperand &, cudaStream_t);
template cudaError_t umma_prep_tn_b<float2>(const void *, int64_t, int64_t, int, UmmaOperand &, cudaStream_t);
template cudaError_t umma_prep_tn_b<double2>(const void *, int64_t, int64_t, int, UmmaOperand &, cudaStream_t);
template cudaError_t umma_prep_nn_a<float2>(const void *, int64_t, int64_t, int, UmmaOperand &, cudaStream_t);
template cudaError_t umma_gemm<float2>(const UmmaOperand &, const UmmaOperand &, int, int, void *, int64_t, int, float *,
                                       int *, cudaStream_t, int, int, int);
template cudaError_t umma_gemm<double2>(const UmmaOperand &, const UmmaOperand &, int, int, void *, int64_t, int, float *,
                                        int *, cudaStream_t, int, int, int);

}  // namespace pwk
