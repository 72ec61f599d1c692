// pw_autotune: picks a context's launch parameters (pw_tuning) by timing
// candidates on the device, with an optional on-disk cache of earlier choices.
//
// The reference has no counterpart: FFTW's planner (PWGrid.jl:98-99,128-129
// plan_fft!/plan_ifft! with the default FFTW.ESTIMATE flags) and the BLAS
// choose their own blockings.  Here the knobs are the band batch of the FFT
// intermediate, the bands per CTA of the FP32 plane pass, the columns per CTA
// of the z passes and the split-K of the tensor-core Rayleigh-Ritz products.
// The tuner is a client of the library's own C ABI (pw_apply, pw_gram,
// pw_rotate, pw_get/set_tuning): what it times is exactly what callers run.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pwb200.h"
#include "pw_launch.h"
#include "pw_tune_cache.h"

cudaStream_t pwk_stream(pw_ctx *c);
int pwk_device(const pw_ctx *c);
int pwk_ngw(const pw_ctx *c, int ik);
int pwk_tune_shape(const pw_ctx *c, int ik, int *Ns, int *Ncol, int *Nxa, int *nbeta);
int pwk_fail_msg(pw_ctx *c, int code, const char *msg);

namespace {

// deterministic fill in [-0.5, 0.5) (the values only have to be finite)
__global__ void k_fill(float *p, size_t n, uint32_t seed) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t h = (uint32_t)i * 2654435761u ^ seed;
        h ^= h >> 16;
        h *= 2246822519u;
        h ^= h >> 13;
        p[i] = (float)(h & 0xffffff) * (1.0f / 16777216.0f) - 0.5f;
    }
}
__global__ void k_f2d(const float *in, double *out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

struct Bufs {
    std::vector<void *> p;
    ~Bufs() {
        for (void *q : p) cudaFree(q);
    }
    void *get(size_t bytes) {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
        p.push_back(q);
        return q;
    }
};

// median device time (ms) of `reps` runs of f() after `warm` untimed ones;
// negative if a run failed
template <class F>
double time_ms(cudaStream_t st, F &&f, int warm = 2, int reps = 5) {
    for (int i = 0; i < warm; ++i)
        if (f() != PW_OK) return -1.0;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<float> ts;
    bool ok = true;
    for (int i = 0; i < reps && ok; ++i) {
        cudaEventRecord(a, st);
        ok = f() == PW_OK;
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        ts.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (!ok || cudaGetLastError() != cudaSuccess) return -1.0;
    std::sort(ts.begin(), ts.end());
    return ts[ts.size() / 2];
}

}  // namespace

extern "C" int pw_autotune(pw_ctx *c, int ik, int nb, int dtype, const char *cache_path, pw_tuning *chosen,
                           double *ms) {
    if (!c) return PW_ERR_ARG;
    int Ns[3], Ncol = 0, Nxa = 0, nbeta = 0;
    if (pwk_tune_shape(c, ik, Ns, &Ncol, &Nxa, &nbeta) != PW_OK)
        return pwk_fail_msg(c, PW_ERR_ARG, "pw_autotune: k-point index out of range");
    if (nb <= 0 || (dtype != PW_C128 && dtype != PW_C64)) return pwk_fail_msg(c, PW_ERR_ARG, "pw_autotune: bad nb or dtype");
    if (ms)
        for (int i = 0; i < 4; ++i) ms[i] = -1.0;
    const int dev = pwk_device(c);
    if (cudaSetDevice(dev) != cudaSuccess) return pwk_fail_msg(c, PW_ERR_CUDA, "cudaSetDevice failed");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return pwk_fail_msg(c, PW_ERR_CUDA, "cudaGetDeviceProperties failed");
    const int ngw = pwk_ngw(c, ik);
    const std::string key = pwk::tune::cache_key(prop.name, Ns, ngw, Ncol, Nxa, nb, dtype, nbeta);
    const char *path = cache_path ? cache_path : std::getenv("PW_AUTOTUNE_CACHE");
    pw_tuning t;
    if (pwk::tune::read_cache(path, key, &t)) {
        int s = pw_set_tuning(c, &t);
        if (s) return s;
        pw_get_tuning(c, &t);   // the values in effect (a zero field reads as its default)
        if (chosen) *chosen = t;
        return PW_OK;
    }
    pw_tuning base;
    pw_get_tuning(c, &base);
    cudaStream_t st = pwk_stream(c);
    const bool f32 = dtype == PW_C64;
    const size_t es = f32 ? 8 : 16;
    const unsigned ops = nbeta > 0 ? PW_OP_H : (PW_OP_K | PW_OP_VLOC);
    Bufs B;
    void *psi = B.get((size_t)nb * ngw * es), *hpsi = B.get((size_t)nb * ngw * es);
    if (!psi || !hpsi) return pwk_fail_msg(c, PW_ERR_NOMEM, "pw_autotune: no device memory for the trial blocks");
    k_fill<<<592, 256, 0, st>>>((float *)psi, (size_t)nb * ngw * es / 4, 12345u);
    auto run_h = [&]() { return pw_apply(c, ik, 0, dtype, psi, hpsi, ngw, nb, ops); };
    auto eval = [&](const pw_tuning &cand) -> double {
        if (pw_set_tuning(c, &cand) != PW_OK) return -1.0;
        return time_ms(st, run_h);
    };
    // ---- op_H: coordinate descent over plane bands, band batch, z columns,
    // from the built-in defaults (whatever the context was set to before)
    pw_tuning best;
    std::memset(&best, 0, sizeof(best));
    double tbest = eval(best);
    if (tbest < 0) {
        pw_set_tuning(c, &base);
        return pwk_fail_msg(c, PW_ERR_STATE, "pw_autotune: op_H failed with the default tuning (is V_loc set?)");
    }
    const double tdef = tbest;
    auto try_field = [&](auto setter, const std::vector<int64_t> &vals) {
        pwk::tune::descend(best, tbest, eval, setter, vals);
    };
    if (f32 && Ns[0] == Ns[1] && (Ns[0] == 27 || Ns[0] == 75 || Ns[0] == 120))
        try_field([](pw_tuning &x, int64_t v) { x.plane_bands = (int32_t)v; }, {1, 2, 3});
    try_field([](pw_tuning &x, int64_t v) { x.band_chunk_bytes = v << 20; }, {16, 24, 32, 48, 72, 96});
    if (f32)
        try_field([](pw_tuning &x, int64_t v) { x.z_columns = (int32_t)v; }, {32, 48, 64, 96, 128});
    else
        try_field([](pw_tuning &x, int64_t v) { x.z_columns = (int32_t)v; }, {16, 24, 32, 48});
    if (ms) {
        ms[0] = tdef;
        ms[1] = tbest;
    }
    // ---- Rayleigh-Ritz products (tensor cores): split-K
    if (f32) {
        const int m = 3 * nb;
        void *Q = B.get((size_t)m * ngw * 8), *C = B.get((size_t)m * m * 16), *U = B.get((size_t)m * nb * 16),
             *Uf = B.get((size_t)m * nb * 16), *out = B.get((size_t)nb * ngw * 8);
        if (Q && C && U && Uf && out) {
            k_fill<<<592, 256, 0, st>>>((float *)Q, (size_t)m * ngw * 2, 777u);
            k_fill<<<592, 256, 0, st>>>((float *)Uf, (size_t)m * nb * 2, 999u);
            k_f2d<<<592, 256, 0, st>>>((const float *)Uf, (double *)U, (size_t)m * nb * 2);
            auto run_rr = [&]() {
                int s = pw_gram(c, PW_C64, ngw, m, m, Q, ngw, Q, ngw, (double *)C, m, 0);
                if (s) return s;
                return pw_rotate(c, PW_C64, ngw, nb, m, Q, ngw, (const double *)U, m, out, ngw, 0);
            };
            double gbest = -1.0, gdef = -1.0;
            int sbest = 0;
            for (int sp : {0, 1, 2, 4, 8, 16, 32}) {
                pw_tuning cand = best;
                cand.gemm_splits = sp;
                if (pw_set_tuning(c, &cand) != PW_OK) continue;
                const double tm = time_ms(st, run_rr);
                if (sp == 0) gdef = tm;
                if (tm > 0 && (gbest < 0 || pwk::tune::faster(tm, gbest))) {
                    gbest = tm;
                    sbest = sp;
                }
            }
            best.gemm_splits = sbest;
            if (ms) {
                ms[2] = gdef;
                ms[3] = gbest;
            }
        }
    }
    cudaStreamSynchronize(st);
    cudaGetLastError();
    int s = pw_set_tuning(c, &best);
    if (s) return s;
    pw_get_tuning(c, &best);    // the values in effect (a zero field reads as its default)
    pwk::tune::append_cache(path, key, best);
    if (chosen) *chosen = best;
    return PW_OK;
}
