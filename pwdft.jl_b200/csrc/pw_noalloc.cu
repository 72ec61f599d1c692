// pw_apply_vloc_noalloc: the op_V_loc (+ op_K) round trip of pw_apply with
// its band-batch intermediate held in a fixed, file-scope device array
// instead of memory the context allocates.  For callers that must not call
// cudaMalloc/cudaFree on this path (see include/pwb200.h).
#include <algorithm>
#include <mutex>

#include "../../include/pwb200.h"
#include "pw_launch.h"

// Upper bound of the scratch: every GPU that loads libpwb200.so holds these
// bytes until the process exits.  Bands are processed in batches that fit;
// a grid whose single band needs more is rejected.
#define PW_NOALLOC_SCRATCH_BYTES (32ull << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[PW_NOALLOC_SCRATCH_BYTES];

int pwk_fail(pw_ctx *c, int code, const char *msg);
void pwk_count_launches(pw_ctx *c, int n);
int pwk_vloc_view(pw_ctx *c, int ik, int ispin, int dtype, pwk::FftLaunch *L, const void **V, cudaStream_t *st,
                  size_t *per_band, int *device);
int pwk_ngw(const pw_ctx *c, int ik);

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};

// The device address of g_noalloc_scratch on `dev` (which must be the current
// device).  Host code cannot use the symbol itself: it names a host-side
// stand-in, not device memory.  The lookup also loads the array's module on
// that device (under CUDA's lazy module loading this is the moment its bytes
// are reserved), so pw_create calls it with refresh = true for its device:
// the reservation happens when a context is built, not on the first
// allocation-free call, and a context built after a device reset records the
// new address.
int lookup_scratch(int dev, bool refresh, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return PW_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    if (refresh || !g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            g_scratch_addr[dev] = nullptr;
            return PW_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return PW_OK;
}

int scratch_address(pw_ctx *c, int dev, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return pwk_fail(c, PW_ERR_ARG, "device index beyond the no-alloc table");
    if (lookup_scratch(dev, false, out) != PW_OK)
        return pwk_fail(c, PW_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch) failed");
    return PW_OK;
}

}  // namespace

// Called by pw_create with `dev` current: reserves the array on that device
// now.  A failure here is not fatal to the context; the allocation-free
// entry point then reports it when it is called.
void pwk_noalloc_prepare(int dev) {
    void *p = nullptr;
    (void)lookup_scratch(dev, true, &p);
}

namespace {

template <typename T>
int run(pw_ctx *c, const pwk::FftLaunch &L, const void *V, cudaStream_t st, void *A, size_t per_band, const void *psi,
        void *Hpsi, int64_t ld, int nb, int flags) {
    const size_t es = 2 * sizeof(T);
    // bands are blockIdx.y of the z passes: at most 65535 per batch
    const int nbc = (int)std::min<size_t>(PW_NOALLOC_SCRATCH_BYTES / per_band, 65535);
    for (int b0 = 0; b0 < nb; b0 += nbc) {
        const int cnt = nb - b0 < nbc ? nb - b0 : nbc;
        const char *pin = (const char *)psi + (size_t)b0 * ld * es;
        char *pout = (char *)Hpsi + (size_t)b0 * ld * es;
        if (pwk::launch_zinv<T>(L, pin, ld, cnt, A, st) != cudaSuccess ||
            pwk::launch_plane_vloc<T>(L, V, A, cnt, st) != cudaSuccess ||
            pwk::launch_zfwd<T>(L, A, pin, pout, ld, cnt, flags, st) != cudaSuccess)
            return pwk_fail(c, PW_ERR_CUDA, "kernel launch failed in pw_apply_vloc_noalloc");
        pwk_count_launches(c, 3);
    }
    return PW_OK;
}

}  // namespace

extern "C" uint64_t pw_noalloc_scratch_bytes(void) { return PW_NOALLOC_SCRATCH_BYTES; }

extern "C" int pw_apply_vloc_noalloc(pw_ctx *c, int ik, int ispin, int dtype, const void *psi, void *Hpsi, int64_t ld,
                                     int nb, unsigned ops) {
    if (!c) return PW_ERR_ARG;
    if (!(ops & PW_OP_VLOC) || (ops & ~(PW_OP_K | PW_OP_VLOC | PW_ACCUMULATE)))
        return pwk_fail(c, PW_ERR_ARG, "pw_apply_vloc_noalloc takes PW_OP_VLOC, optionally with PW_OP_K and PW_ACCUMULATE");
    if (!psi || !Hpsi || psi == Hpsi) return pwk_fail(c, PW_ERR_ARG, "psi and Hpsi must be distinct device buffers");
    pwk::FftLaunch L;
    const void *V = nullptr;
    cudaStream_t st = nullptr;
    size_t per_band = 0;
    int dev = 0;
    int s = pwk_vloc_view(c, ik, ispin, dtype, &L, &V, &st, &per_band, &dev);
    if (s) return s;
    if (nb <= 0 || ld < pwk_ngw(c, ik)) return pwk_fail(c, PW_ERR_ARG, "bad shape (nb <= 0 or ld < Ngw)");
    if (per_band > PW_NOALLOC_SCRATCH_BYTES)
        return pwk_fail(c, PW_ERR_UNSUPPORTED,
                        "one band of this grid needs more than the 32 MiB no-alloc scratch; use pw_apply");
    if (cudaSetDevice(dev) != cudaSuccess) return pwk_fail(c, PW_ERR_CUDA, "cudaSetDevice failed");
    void *A = nullptr;
    if ((s = scratch_address(c, dev, &A))) return s;
    const int flags = ((ops & PW_OP_K) ? 2 : 0) | ((ops & PW_ACCUMULATE) ? 4 : 0);
    return dtype == PW_C128 ? run<double>(c, L, V, st, A, per_band, psi, Hpsi, ld, nb, flags)
                            : run<float>(c, L, V, st, A, per_band, psi, Hpsi, ld, nb, flags);
}
