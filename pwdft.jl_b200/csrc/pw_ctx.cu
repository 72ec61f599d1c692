// Context, set-up and the C ABI of libpwb200.so (declared in include/pwb200.h).
//
// The context replaces what PWDFT.jl keeps in Ham.pw (FFTW plans, index
// maps), Ham.potentials.Total and Ham.pspotNL for the operators; the
// kernels themselves live in pw_fft_kernels.cu and pw_gemm.cu.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pwb200.h"
#include "pw_launch.h"
#include "pw_umma.h"

using namespace pwk;

void pwk_noalloc_prepare(int dev);   // pw_noalloc.cu
void pwk_mix_free(void *state);      // pw_mix.cu

namespace {

thread_local std::string g_create_error;

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct KData {
    int Ngw = 0, Ncol = 0, Nxa = 0;
    int *d_col_ptr = nullptr, *d_ent_igw = nullptr, *d_ent_kz = nullptr, *d_ent_col = nullptr;
    int *d_col_ia = nullptr, *d_col_j = nullptr, *d_xa = nullptr;
    double *d_Gk2 = nullptr;
    float *d_Gk2f = nullptr;
    double *d_eg2 = nullptr;   // |G+k|^2 in entry order
    float *d_eg2f = nullptr;
    double2 *d_beta64 = nullptr;
    float2 *d_beta32 = nullptr;
    UmmaOperand beta_tn;  // split-BF16 betaNL for betaNL' psi   (tensor-core path)
    UmmaOperand beta_nn;  // split-BF16 betaNL^H for betaNL * P  (tensor-core path)
    double *d_gk = nullptr;  // (G+k) vectors, 3 x Ngw (forces)
};

constexpr int kMaxV64 = 8;  // complex values per thread per round in the FP64 FFT stages
constexpr int kFftThreads = 256;

bool make_plan(int n, FftDim &d) {
    d.n = n;
    d.nstage = 0;
    int m = n;
    const int radices[5] = {8, 4, 2, 3, 5};
    for (int r : radices) {
        while (m % r == 0) {
            if (d.nstage >= 12) return false;
            const int maxb = std::max(1, kMaxV64 / r);
            if (n / r > 32 * maxb) return false;  // one warp must hold a whole line stage
            d.radix[d.nstage++] = r;
            m /= r;
        }
    }
    return m == 1;
}

}  // namespace

struct pw_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int N1 = 0, N2 = 0, N3 = 0;
    size_t N = 0;
    int Nkpt = 0, Nspin = 1;
    double CellVolume = 0;
    FftDim dx{}, dy{}, dz{};
    double2 *tw64[3] = {nullptr, nullptr, nullptr};
    float2 *tw32[3] = {nullptr, nullptr, nullptr};
    std::vector<KData> k;
    double *d_V64 = nullptr;
    float *d_V32 = nullptr;
    int vloc_nspin = 0;
    int nbeta = 0;
    int *d_Drow = nullptr, *d_Dcol = nullptr;
    double *d_Dval = nullptr;
    bool have_D = false;
    DevBuf A, P, P2, gemm_ws, rho_part, w, st_in, st_out, st_in32, st_out32, st_rho;
    std::vector<void *> allocs;
    size_t a_chunk_bytes = 48ull << 20;
    int plane_bpc = 0;        // bands per CTA of the FP32 plane kernels (0: per-grid default)
    int z_cols = 0;           // columns per CTA of the z passes (0: the 48 KB default)
    int gemm_splits = 0;      // split-K of the tensor-core GEMMs (0: automatic)
    bool use_umma = true;     // mixed-precision contractions on tcgen05 (PW_GEMM=cuda: CUDA cores)
    int *d_err = nullptr;     // device error word of the bounded waits in the tensor-core kernels
    DevBuf um_a_hi, um_a_lo, um_b_hi, um_b_lo, um_b_lo2, um_ws;
    DevBuf slots[32];         // grow-only scratch for the eigensolver and LOBPCG
    KData dens;               // the density G-sphere (for Poisson_solve! on the device)
    bool have_dens = false;
    // forces: G vectors of the density sphere (3 x Ng), V_sp(G) per species
    // (Ng x nspecies), projector rows of each atom (natoms + 1 offsets)
    double *d_fG = nullptr, *d_fV = nullptr;
    int f_nsp = 0;
    int *d_atom_rows = nullptr;
    int f_natoms = 0;
    // exchange-correlation of update!: PW_XC_VWN or PW_XC_PBE (with the G
    // vectors of the density sphere, 3 x Ng, for grad rho and div h)
    int xc = PW_XC_VWN;
    double *d_xcG = nullptr;
    // batched op_H over k-points: device tables (MkK per k-point, band ->
    // k-point map), and the CUDA graph of the last call made with PW_GRAPH
    // symmetrize_rhoe!: orbits of the density sphere (nshell x nsym sphere
    // indices and phases e^{i G.ft})
    int *d_sym_isg = nullptr;
    double2 *d_sym_ph = nullptr;
    int sym_nshell = 0, sym_nsym = 0;
    DevBuf mk_tab;
    uint64_t mk_key = 0;
    cudaGraphExec_t mk_exec = nullptr;
    int mk_nlaunch = 0;

    cudaStream_t cap_stream = nullptr;
    // host drop-ins: copy streams and per-chunk events of the pipelined op_H
    cudaStream_t cp_in = nullptr, cp_out = nullptr;
    cudaEvent_t ev_in[8] = {}, ev_cmp[8] = {};
    int64_t launches = 0;  // kernels launched by this context (reported by pw_launch_count)
    void *mix_state = nullptr;  // Pulay history of pw_mix_pulay (pw_mix.cu)
};

namespace {

int fail(pw_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c)
        c->err = buf;
    else
        g_create_error = buf;
    return code;
}

#define CK(ctx, x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) return fail(ctx, PW_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int dalloc(pw_ctx *c, T **p, size_t n) {
    void *q = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return fail(c, PW_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    c->allocs.push_back(q);
    *p = (T *)q;
    return PW_OK;
}

template <typename T>
int upload(pw_ctx *c, T **p, const std::vector<T> &v) {
    int s = dalloc(c, p, v.size());
    if (s) return s;
    CK(c, cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PW_OK;
}

void dfree(pw_ctx *c, void *p) {
    if (!p) return;
    auto it = std::find(c->allocs.begin(), c->allocs.end(), p);
    if (it != c->allocs.end()) c->allocs.erase(it);
    cudaFree(p);
}

int ensure(pw_ctx *c, DevBuf &b, size_t bytes) {
    if (b.bytes >= bytes) return PW_OK;
    if (b.p) {
        cudaStreamSynchronize(c->stream);
        dfree(c, b.p);
        b.p = nullptr;
        b.bytes = 0;
    }
    void *q = nullptr;
    int s = dalloc(c, (unsigned char **)&q, bytes);
    if (s) return s;
    b.p = q;
    b.bytes = bytes;
    return PW_OK;
}

int build_twiddles(pw_ctx *c, int n, int slot) {
    std::vector<double2> t64(n);
    std::vector<float2> t32(n);
    for (int m = 0; m < n; ++m) {
        const double a = -2.0 * M_PI * (double)m / (double)n;
        t64[m] = make_double2(std::cos(a), std::sin(a));
        t32[m] = make_float2((float)t64[m].x, (float)t64[m].y);
    }
    int s = upload(c, &c->tw64[slot], t64);
    if (s) return s;
    return upload(c, &c->tw32[slot], t32);
}

// Builds the pruned-FFT tables of one k-point from its sphere -> grid map.
int build_kdata(pw_ctx *c, KData &kd, int64_t Ngw, const int64_t *idx, int base, const double *Gk2) {
    const int N1 = c->N1, N2 = c->N2, N3 = c->N3;
    const int64_t N = (int64_t)c->N;
    if (Ngw <= 0 || Ngw > (int64_t)INT32_MAX) return fail(c, PW_ERR_ARG, "Ngw out of range: %lld", (long long)Ngw);
    kd.Ngw = (int)Ngw;
    std::vector<int> ent_i(Ngw), ent_j(Ngw), ent_k(Ngw);
    std::vector<unsigned char> seen(N, 0);
    for (int64_t g = 0; g < Ngw; ++g) {
        const int64_t ip = idx[g] - base;
        if (ip < 0 || ip >= N) return fail(c, PW_ERR_ARG, "idx_gw2r[%lld] = %lld outside the grid", (long long)g, (long long)idx[g]);
        if (seen[ip]) return fail(c, PW_ERR_ARG, "idx_gw2r maps two G-vectors onto grid point %lld", (long long)ip);
        seen[ip] = 1;
        ent_i[g] = (int)(ip % N1);
        ent_j[g] = (int)((ip / N1) % N2);
        ent_k[g] = (int)(ip / ((int64_t)N1 * N2));
    }
    // active columns, x-major (all columns of one x are adjacent)
    std::vector<int> colid((size_t)N1 * N2, -1);
    for (int64_t g = 0; g < Ngw; ++g) colid[(size_t)ent_i[g] * N2 + ent_j[g]] = 0;
    std::vector<int> col_i, col_j;
    for (int i = 0; i < N1; ++i)
        for (int j = 0; j < N2; ++j)
            if (colid[(size_t)i * N2 + j] == 0) {
                colid[(size_t)i * N2 + j] = (int)col_i.size();
                col_i.push_back(i);
                col_j.push_back(j);
            }
    const int Ncol = (int)col_i.size();
    std::vector<int> col_ptr(Ncol + 1, 0);
    std::vector<int> ecol(Ngw);
    for (int64_t g = 0; g < Ngw; ++g) {
        ecol[g] = colid[(size_t)ent_i[g] * N2 + ent_j[g]];
        col_ptr[ecol[g] + 1]++;
    }
    for (int cc = 0; cc < Ncol; ++cc) col_ptr[cc + 1] += col_ptr[cc];
    std::vector<int> order(Ngw);
    for (int64_t g = 0; g < Ngw; ++g) order[g] = (int)g;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return ecol[a] != ecol[b] ? ecol[a] < ecol[b] : ent_k[a] < ent_k[b];
    });
    std::vector<int> e_igw(Ngw), e_kz(Ngw), e_col(Ngw);
    for (int64_t e = 0; e < Ngw; ++e) {
        e_igw[e] = order[e];
        e_kz[e] = ent_k[order[e]];
        e_col[e] = ecol[order[e]];
    }
    std::vector<int> xa, col_ia(Ncol);
    for (int cc = 0; cc < Ncol; ++cc) {
        if (xa.empty() || xa.back() != col_i[cc]) xa.push_back(col_i[cc]);
        col_ia[cc] = (int)xa.size() - 1;
    }
    kd.Ncol = Ncol;
    kd.Nxa = (int)xa.size();
    int s;
    if ((s = upload(c, &kd.d_col_ptr, col_ptr))) return s;
    if ((s = upload(c, &kd.d_ent_igw, e_igw))) return s;
    if ((s = upload(c, &kd.d_ent_kz, e_kz))) return s;
    if ((s = upload(c, &kd.d_ent_col, e_col))) return s;
    if ((s = upload(c, &kd.d_col_ia, col_ia))) return s;
    if ((s = upload(c, &kd.d_col_j, col_j))) return s;
    if ((s = upload(c, &kd.d_xa, xa))) return s;
    std::vector<double> g2(Gk2, Gk2 + Ngw);
    std::vector<float> g2f(Ngw);
    for (int64_t g = 0; g < Ngw; ++g) g2f[g] = (float)g2[g];
    if ((s = upload(c, &kd.d_Gk2, g2))) return s;
    if ((s = upload(c, &kd.d_Gk2f, g2f))) return s;
    std::vector<double> eg2(Ngw);
    std::vector<float> eg2f(Ngw);
    for (int64_t e = 0; e < Ngw; ++e) {
        eg2[e] = g2[e_igw[e]];
        eg2f[e] = g2f[e_igw[e]];
    }
    if ((s = upload(c, &kd.d_eg2, eg2))) return s;
    if ((s = upload(c, &kd.d_eg2f, eg2f))) return s;
    (void)N3;
    return PW_OK;
}

template <typename T>
FftLaunch make_launch_kd(const pw_ctx *c, const KData &kd);

template <typename T>
FftLaunch make_launch(const pw_ctx *c, int ik) {
    return make_launch_kd<T>(c, c->k[ik]);
}

template <typename T>
FftLaunch make_launch_kd(const pw_ctx *c, const KData &kd) {
    FftLaunch L;
    L.kp.N1 = c->N1;
    L.kp.N2 = c->N2;
    L.kp.N3 = c->N3;
    L.kp.Ngw = kd.Ngw;
    L.kp.Ncol = kd.Ncol;
    L.kp.Nxa = kd.Nxa;
    L.kp.col_ptr = kd.d_col_ptr;
    L.kp.ent_igw = kd.d_ent_igw;
    L.kp.ent_kz = kd.d_ent_kz;
    L.kp.ent_col = kd.d_ent_col;
    L.kp.col_ia = kd.d_col_ia;
    L.kp.col_j = kd.d_col_j;
    L.kp.xa = kd.d_xa;
    L.kp.Gk2 = kd.d_Gk2;
    L.kp.Gk2f = kd.d_Gk2f;
    L.kp.ent_g2 = kd.d_eg2;
    L.kp.ent_g2f = kd.d_eg2f;
    L.dx = c->dx;
    L.dy = c->dy;
    L.dz = c->dz;
    const bool dbl = sizeof(T) == 8;
    L.twx = dbl ? (const void *)c->tw64[0] : (const void *)c->tw32[0];
    L.twy = dbl ? (const void *)c->tw64[1] : (const void *)c->tw32[1];
    L.twz = dbl ? (const void *)c->tw64[2] : (const void *)c->tw32[2];
    const size_t es = 2 * sizeof(T);
    // z passes: ~48 KB of shared memory per CTA
    int Cg = (int)((48 * 1024 / es - c->N3) / c->N3);
    L.Cg = std::max(1, std::min(64, Cg));
    if (c->z_cols > 0) {
        // at most ~190 KB of shared memory per z-pass CTA
        const int cmax = std::max(1, (int)((190 * 1024 / es - c->N3) / c->N3) - 16);
        L.Cg = std::min(c->z_cols, cmax);
    }
    L.bpc = c->plane_bpc > 0 ? c->plane_bpc : (c->N1 == 75 ? 3 : 1);
    // plane passes: a 100 KB budget (two CTAs per SM) when it holds at
    // least 16 full x lines, otherwise up to 220 KB
    const size_t fixed = (size_t)c->N1 + c->N2 + (size_t)kd.Nxa * c->N2;
    size_t budget = 100 * 1024 / es;
    if (budget < fixed + (size_t)std::min(16, c->N2) * c->N1) budget = 220 * 1024 / es;
    long Jc = budget > fixed ? (long)((budget - fixed) / c->N1) : 0;
    L.Jc = (int)std::max(1L, std::min((long)c->N2, Jc));
    return L;
}

size_t plane_smem_bytes(const pw_ctx *c, const FftLaunch &L, size_t es) {
    return ((size_t)c->N1 + c->N2 + (size_t)L.kp.Nxa * c->N2 + (size_t)L.Jc * c->N1) * es;
}

int check_k(pw_ctx *c, int ik) {
    if (ik < 0 || ik >= c->Nkpt) return fail(c, PW_ERR_ARG, "k-point index %d outside [0, %d)", ik, c->Nkpt);
    return PW_OK;
}

int band_chunk(const pw_ctx *c, int ik, size_t es, int nb) {
    const size_t per_band = (size_t)c->N3 * c->k[ik].Ncol * es;
    size_t ch = c->a_chunk_bytes / std::max<size_t>(per_band, 1);
    if (ch < 1) ch = 1;
    if (ch > 65535) ch = 65535;   // bands are blockIdx.y of the z passes
    return (int)std::min<size_t>(ch, (size_t)nb);
}

// Per-call split-BF16 operands live in grow-only scratch buffers (lo2: a
// third BF16 piece, for the products that need ~2^-24).
int umma_scratch(pw_ctx *c, DevBuf &hi, DevBuf &lo, int64_t rows, int64_t K, UmmaOperand &op, DevBuf *lo2 = nullptr) {
    const size_t half = umma_operand_bytes(rows, K) / 2;
    int s;
    if ((s = ensure(c, hi, half)) || (s = ensure(c, lo, half))) return s;
    op.hi = (__nv_bfloat16 *)hi.p;
    op.lo = (__nv_bfloat16 *)lo.p;
    op.lo2 = nullptr;
    if (lo2) {
        if ((s = ensure(c, *lo2, half))) return s;
        op.lo2 = (__nv_bfloat16 *)lo2->p;
    }
    return PW_OK;
}

// C (m x n, CT) (+)= Z^H W  on tensor cores; Z, W complex64 (K x m / K x n).
template <typename CT>
int umma_tn(pw_ctx *c, int64_t K, int m, int n, const void *Z, int64_t ldz, const void *Wm, int64_t ldw, void *C,
            int64_t ldc, int acc, int upper = 0) {
    UmmaOperand A, B;
    int s;
    const int same = (Z == Wm && ldz == ldw && m == n);   // Z^H Z: add the lo*lo product
    if ((s = umma_scratch(c, c->um_a_hi, c->um_a_lo, 2 * (int64_t)m, K, A))) return s;
    CK(c, umma_prep_tn_a<float2>(Z, ldz, K, m, A, c->stream));
    if (same) {
        // the B' rows [Re z_j, Im z_j] of Z^H Z are the even rows of A'
        B = A;
        B.rows = n;
        B.rstride = 2;
    } else {
        if ((s = umma_scratch(c, c->um_b_hi, c->um_b_lo, n, K, B))) return s;
        CK(c, umma_prep_tn_b<float2>(Wm, ldw, K, n, B, c->stream));
    }
    if ((s = ensure(c, c->um_ws, umma_ws_bytes(A.rows, n, A.Kp, c->gemm_splits, upper)))) return s;
    CK(c, umma_gemm<CT>(A, B, m, n, C, ldc, acc, (float *)c->um_ws.p, c->d_err, c->stream, upper, same, c->gemm_splits));
    c->launches += (same ? 2 : 3) + (acc || umma_splits(A.rows, n, A.Kp, c->gemm_splits, upper) > 1 ? 1 : 0);
    return PW_OK;
}

// C (M x n, complex64) (+)= A (M x k, complex64) U (k x n, complex128) on tensor cores.
int umma_nn(pw_ctx *c, int64_t M, int n, int k, const void *A, int64_t lda, const UmmaOperand *Aprep, const double2 *U,
            int64_t ldu, void *C, int64_t ldc, int acc) {
    UmmaOperand Ao, B;
    int s;
    if (Aprep) {
        Ao = *Aprep;
    } else {
        if ((s = umma_scratch(c, c->um_a_hi, c->um_a_lo, 2 * M, k, Ao))) return s;
        CK(c, umma_prep_nn_a<float2>(A, lda, M, k, Ao, c->stream));
        c->launches += 2;
    }
    if ((s = umma_scratch(c, c->um_b_hi, c->um_b_lo, n, k, B))) return s;
    CK(c, umma_prep_tn_b<double2>(U, ldu, k, n, B, c->stream));
    if ((s = ensure(c, c->um_ws, umma_ws_bytes(Ao.rows, n, Ao.Kp, c->gemm_splits)))) return s;
    CK(c, umma_gemm<float2>(Ao, B, (int)M, n, C, ldc, acc, (float *)c->um_ws.p, c->d_err, c->stream, 0, 0,
                            c->gemm_splits));
    c->launches += 2 + (acc || umma_splits(Ao.rows, n, Ao.Kp, c->gemm_splits) > 1 ? 1 : 0);
    return PW_OK;
}

template <typename T>
int apply_T(pw_ctx *c, int ik, int ispin, const void *psi, void *Hpsi, int64_t ld, int nb, unsigned ops) {
    const KData &kd = c->k[ik];
    const unsigned o = ops & PW_OP_H;
    const int acc = (ops & PW_ACCUMULATE) ? 1 : 0;
    const size_t es = 2 * sizeof(T);
    cudaStream_t st = c->stream;
    const void *beta = sizeof(T) == 8 ? (const void *)kd.d_beta64 : (const void *)kd.d_beta32;
    if (o & PW_OP_VNL) {
        if (c->nbeta <= 0 || !beta || !c->have_D)
            return fail(c, PW_ERR_STATE, "op_V_Ps_nloc requested but the projectors of k-point %d are not set", ik);
        int s;
        const size_t pb = (size_t)c->nbeta * nb * sizeof(double2);
        if ((s = ensure(c, c->P, pb)) || (s = ensure(c, c->P2, pb))) return s;
        if (sizeof(T) == 4 && c->use_umma) {
            // betaNL' psi cancels heavily (|beta' psi| << |beta||psi|): three
            // BF16 pieces keep its error at FP32 level; two bias <psi|V_NL|psi>
            UmmaOperand B;
            if ((s = umma_scratch(c, c->um_b_hi, c->um_b_lo, nb, kd.Ngw, B, &c->um_b_lo2))) return s;
            CK(c, umma_prep_tn_b<float2>(psi, ld, kd.Ngw, nb, B, st));
            if ((s = ensure(c, c->um_ws, umma_ws_bytes(kd.beta_tn.rows, nb, kd.beta_tn.Kp)))) return s;
            CK(c, umma_gemm<double2>(kd.beta_tn, B, c->nbeta, nb, c->P.p, c->nbeta, 0, (float *)c->um_ws.p, c->d_err, st));
            c->launches += 2 + (umma_splits(kd.beta_tn.rows, nb, kd.beta_tn.Kp) > 1 ? 1 : 0);
        } else {
            if ((s = ensure(c, c->gemm_ws, gemm_tn_ws_bytes(kd.Ngw, c->nbeta, nb)))) return s;
            CK(c, (gemm_tn<T>(kd.Ngw, c->nbeta, nb, beta, kd.Ngw, psi, ld, (double2 *)c->P.p, c->nbeta, 0, c->gemm_ws.p, st)));
            c->launches += 2;
        }
        CK(c, apply_dcsr(c->nbeta, nb, c->d_Drow, c->d_Dcol, c->d_Dval, (const double2 *)c->P.p, (double2 *)c->P2.p, st));
        c->launches += 1;
    }
    if (o & PW_OP_VLOC) {
        if (c->vloc_nspin <= 0) return fail(c, PW_ERR_STATE, "op_V_loc requested before pw_set_vloc");
        if (ispin < 0 || ispin >= c->vloc_nspin) return fail(c, PW_ERR_ARG, "spin index %d outside [0, %d)", ispin, c->vloc_nspin);
        FftLaunch L = make_launch<T>(c, ik);
        const int nbc = band_chunk(c, ik, es, nb);
        int s;
        if ((s = ensure(c, c->A, (size_t)nbc * c->N3 * kd.Ncol * es))) return s;
        const void *V = sizeof(T) == 8 ? (const void *)(c->d_V64 + (size_t)ispin * c->N)
                                       : (const void *)(c->d_V32 + (size_t)ispin * c->N);
        const int flags = ((o & PW_OP_K) ? 2 : 0) | (acc ? 4 : 0);
        for (int b0 = 0; b0 < nb; b0 += nbc) {
            const int cnt = std::min(nbc, nb - b0);
            const char *pin = (const char *)psi + (size_t)b0 * ld * es;
            char *pout = (char *)Hpsi + (size_t)b0 * ld * es;
            CK(c, launch_zinv<T>(L, pin, ld, cnt, c->A.p, st));
            CK(c, launch_plane_vloc<T>(L, V, c->A.p, cnt, st));
            CK(c, launch_zfwd<T>(L, c->A.p, pin, pout, ld, cnt, flags, st));
            c->launches += 3;
        }
    } else if (o & PW_OP_K) {
        CK(c, launch_opK<T>(kd.Ngw, nb, kd.d_Gk2, psi, Hpsi, ld, acc, st));
        c->launches += 1;
    } else if (!acc) {
        CK(c, launch_zero<T>(Hpsi, kd.Ngw, nb, ld, st));
        c->launches += 1;
    }
    if (o & PW_OP_VNL) {
        if (sizeof(T) == 4 && c->use_umma) {
            int s;
            if ((s = umma_nn(c, kd.Ngw, nb, c->nbeta, nullptr, 0, &kd.beta_nn, (const double2 *)c->P2.p, c->nbeta, Hpsi,
                             ld, 1)))
                return s;
        } else {
            CK(c, gemm_nn<T>(kd.Ngw, nb, c->nbeta, beta, kd.Ngw, (const double2 *)c->P2.p, c->nbeta, Hpsi, ld, 1, st));
            c->launches += 1;
        }
    }
    return PW_OK;
}

template <typename T>
int rhoe_T(pw_ctx *c, int ik, const void *psi, int64_t ld, int nb, const double *w_host, double *rhoe, int accumulate) {
    const KData &kd = c->k[ik];
    const size_t es = 2 * sizeof(T);
    cudaStream_t st = c->stream;
    FftLaunch L = make_launch<T>(c, ik);
    const int nbc = band_chunk(c, ik, es, nb);
    int s;
    if ((s = ensure(c, c->A, (size_t)nbc * c->N3 * kd.Ncol * es))) return s;
    // band groups: enough CTAs (N3 * G) to fill the GPU twice
    int G = std::max(1, std::min(nbc, (2 * 148 + c->N3 - 1) / c->N3));
    if ((s = ensure(c, c->rho_part, (size_t)G * c->N * sizeof(T)))) return s;
    if ((s = ensure(c, c->w, (size_t)nb * sizeof(double)))) return s;
    std::vector<double> wv(w_host, w_host + nb);
    for (auto &x : wv) x /= c->CellVolume;
    CK(c, cudaMemcpyAsync(c->w.p, wv.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
    for (int b0 = 0; b0 < nb; b0 += nbc) {
        const int cnt = std::min(nbc, nb - b0);
        const int Gc = std::min(G, cnt);
        const int Bg = (cnt + Gc - 1) / Gc;
        const int Gu = (cnt + Bg - 1) / Bg;
        const char *pin = (const char *)psi + (size_t)b0 * ld * es;
        CK(c, launch_zinv<T>(L, pin, ld, cnt, c->A.p, st));
        CK(c, launch_plane_rho<T>(L, c->A.p, cnt, Gu, Bg, (const double *)c->w.p + b0, c->rho_part.p, st));
        CK(c, launch_rho_reduce<T>(c->rho_part.p, Gu, c->N, rhoe, (b0 == 0) ? accumulate : 1, st));
        c->launches += 3;
    }
    // the weights live in a pageable host vector: finish before it goes away
    CK(c, cudaStreamSynchronize(st));
    return PW_OK;
}

int check_dtype(pw_ctx *c, int dtype) {
    if (dtype != PW_C128 && dtype != PW_C64) return fail(c, PW_ERR_ARG, "unknown dtype %d", dtype);
    return PW_OK;
}

}  // namespace

// ====================================================================== ABI

extern "C" int pw_abi_version(void) { return PWB200_ABI_VERSION; }

extern "C" const char *pw_last_error(const pw_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

extern "C" int pw_create(int device, const pw_grid_desc *d, pw_ctx **out) {
    if (!out) return fail(nullptr, PW_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!d) return fail(nullptr, PW_ERR_ARG, "desc is NULL");
    if (d->Ns[0] <= 0 || d->Ns[1] <= 0 || d->Ns[2] <= 0 || d->Nkpt <= 0 || d->Nspin < 1 || d->Nspin > 2 ||
        !(d->CellVolume > 0) || !d->Ngw || !d->idx_gw2r || !d->Gk2 || (d->index_base != 0 && d->index_base != 1))
        return fail(nullptr, PW_ERR_ARG, "invalid grid description");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(nullptr, PW_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(nullptr, PW_ERR_ARG, "device %d outside [0, %d)", device, ndev);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, PW_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    pw_ctx *c = new pw_ctx();
    c->device = device;
    c->N1 = d->Ns[0];
    c->N2 = d->Ns[1];
    c->N3 = d->Ns[2];
    c->N = (size_t)c->N1 * c->N2 * c->N3;
    c->Nkpt = d->Nkpt;
    c->Nspin = d->Nspin;
    c->CellVolume = d->CellVolume;
    if (const char *s = getenv("PW_A_CHUNK_MB")) c->a_chunk_bytes = (size_t)std::max(1, atoi(s)) << 20;
    if (const char *s = getenv("PW_GEMM")) c->use_umma = strcmp(s, "cuda") != 0;
    int st = PW_OK;
    if (!make_plan(c->N1, c->dx) || !make_plan(c->N2, c->dy) || !make_plan(c->N3, c->dz)) {
        st = fail(nullptr, PW_ERR_UNSUPPORTED, "grid %dx%dx%d: every dimension must factor into 2,3,5 and fit one warp per line (<= 160 with a factor 5)",
                  c->N1, c->N2, c->N3);
    }
    if (!st) pwk_noalloc_prepare(device);
    if (!st) {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) st = fail(nullptr, PW_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        c->own_stream = true;
    }
    for (int s = 0; s < 3 && !st; ++s) st = build_twiddles(c, d->Ns[s], s);
    if (!st && !(st = dalloc(c, &c->d_err, 1))) {
        e = cudaMemset(c->d_err, 0, sizeof(int));
        if (e != cudaSuccess) st = fail(c, PW_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    }
    if (!st) {
        c->k.resize(c->Nkpt);
        for (int ik = 0; ik < c->Nkpt && !st; ++ik) {
            if (!d->idx_gw2r[ik] || !d->Gk2[ik]) {
                st = fail(c, PW_ERR_ARG, "k-point %d: NULL idx_gw2r or Gk2", ik);
                break;
            }
            st = build_kdata(c, c->k[ik], d->Ngw[ik], d->idx_gw2r[ik], d->index_base, d->Gk2[ik]);
        }
    }
    if (st) {
        if (!c->err.empty()) g_create_error = c->err;
        pw_destroy(c);
        return st;
    }
    *out = c;
    return PW_OK;
}

extern "C" void pw_destroy(pw_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->mk_exec) cudaGraphExecDestroy(c->mk_exec);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    for (int i = 0; i < 8; ++i) {
        if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
        if (c->ev_cmp[i]) cudaEventDestroy(c->ev_cmp[i]);
    }
    if (c->cp_in) cudaStreamDestroy(c->cp_in);
    if (c->cp_out) cudaStreamDestroy(c->cp_out);
    pwk_mix_free(c->mix_state);
    for (void *p : c->allocs) cudaFree(p);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" int pw_set_stream(pw_ctx *c, void *stream) {
    if (!c) return PW_ERR_ARG;
    if (c->own_stream && c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    c->own_stream = false;
    c->stream = (cudaStream_t)stream;
    return PW_OK;
}

extern "C" int64_t pw_launch_count(const pw_ctx *c) { return c ? c->launches : -1; }

extern "C" int pw_get_tuning(const pw_ctx *c, pw_tuning *t) {
    if (!c || !t) return PW_ERR_ARG;
    std::memset(t, 0, sizeof(*t));
    t->band_chunk_bytes = (int64_t)c->a_chunk_bytes;
    t->plane_bands = c->plane_bpc;
    t->z_columns = c->z_cols;
    t->gemm_splits = c->gemm_splits;
    return PW_OK;
}

extern "C" int pw_set_tuning(pw_ctx *c, const pw_tuning *t) {
    if (!c) return PW_ERR_ARG;
    if (!t) return fail(c, PW_ERR_ARG, "tuning is NULL");
    for (int i = 0; i < 5; ++i)
        if (t->reserved[i]) return fail(c, PW_ERR_ARG, "pw_tuning.reserved[%d] must be zero", i);
    if (t->band_chunk_bytes < 0 || t->plane_bands < 0 || t->plane_bands > 3 || t->z_columns < 0 ||
        t->z_columns > 256 || t->gemm_splits < 0 || t->gemm_splits > 64)
        return fail(c, PW_ERR_ARG, "tuning out of range: chunk %lld, plane_bands %d, z_columns %d, gemm_splits %d",
                    (long long)t->band_chunk_bytes, t->plane_bands, t->z_columns, t->gemm_splits);
    c->a_chunk_bytes = t->band_chunk_bytes > 0 ? (size_t)t->band_chunk_bytes : (48ull << 20);
    c->plane_bpc = t->plane_bands;
    c->z_cols = t->z_columns;
    c->gemm_splits = t->gemm_splits;
    return PW_OK;
}

extern "C" int pw_check_device(pw_ctx *c) {
    if (!c) return PW_ERR_ARG;
    int h = 0;
    CK(c, cudaStreamSynchronize(c->stream));
    CK(c, cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h)
        return fail(c, PW_ERR_TIMEOUT, "a bounded device-side wait expired (code %d: 1-2 tensor-core GEMM pipeline, "
                    "3 grid barrier of the persistent batched op_H)", h);
    return PW_OK;
}

extern "C" int pw_device_alloc(pw_ctx *c, uint64_t bytes, void **dptr) {
    if (!c) return PW_ERR_ARG;
    if (!dptr || bytes == 0) return fail(c, PW_ERR_ARG, "pw_device_alloc: NULL out pointer or zero size");
    CK(c, cudaSetDevice(c->device));
    unsigned char *p = nullptr;
    int s = dalloc(c, &p, (size_t)bytes);
    if (s) return s;
    *dptr = p;
    return PW_OK;
}

extern "C" int pw_device_free(pw_ctx *c, void *dptr) {
    if (!c) return PW_ERR_ARG;
    if (!dptr) return PW_OK;
    if (std::find(c->allocs.begin(), c->allocs.end(), dptr) == c->allocs.end())
        return fail(c, PW_ERR_ARG, "pw_device_free: pointer not from pw_device_alloc of this context");
    CK(c, cudaSetDevice(c->device));
    CK(c, cudaStreamSynchronize(c->stream));
    dfree(c, dptr);
    return PW_OK;
}

extern "C" int pw_copy_to_device(pw_ctx *c, void *dst, const void *src, uint64_t bytes) {
    if (!c) return PW_ERR_ARG;
    if (!dst || !src) return fail(c, PW_ERR_ARG, "pw_copy_to_device: NULL pointer");
    CK(c, cudaSetDevice(c->device));
    CK(c, cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return PW_OK;
}

extern "C" int pw_copy_to_host(pw_ctx *c, void *dst, const void *src, uint64_t bytes) {
    if (!c) return PW_ERR_ARG;
    if (!dst || !src) return fail(c, PW_ERR_ARG, "pw_copy_to_host: NULL pointer");
    CK(c, cudaSetDevice(c->device));
    CK(c, cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return PW_OK;
}

extern "C" int pw_synchronize(pw_ctx *c) {
    if (!c) return PW_ERR_ARG;
    CK(c, cudaStreamSynchronize(c->stream));
    return PW_OK;
}

static int set_vloc_common(pw_ctx *c, const double *V, int nspin, bool on_device) {
    if (!c || !V) return c ? fail(c, PW_ERR_ARG, "V is NULL") : PW_ERR_ARG;
    if (nspin < 1 || nspin > 2) return fail(c, PW_ERR_ARG, "nspin %d not in {1, 2}", nspin);
    CK(c, cudaSetDevice(c->device));
    const size_t n = c->N * nspin;
    if (c->vloc_nspin < nspin) {
        dfree(c, c->d_V64);
        dfree(c, c->d_V32);
        c->d_V64 = nullptr;
        c->d_V32 = nullptr;
        int s;
        if ((s = dalloc(c, &c->d_V64, n)) || (s = dalloc(c, &c->d_V32, n))) return s;
    }
    CK(c, cudaMemcpyAsync(c->d_V64, V, n * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          c->stream));
    // fold the 1/N of G_to_R into the potential: fft(V .* ifft(x)) = fft((V/N) .* bfft(x))
    const double inv = 1.0 / (double)c->N;
    CK(c, convert_d_to_f(c->d_V64, c->d_V32, n, inv, c->stream));
    CK(c, scale_d(c->d_V64, c->d_V64, n, inv, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->vloc_nspin = nspin;
    return PW_OK;
}

extern "C" int pw_set_vloc(pw_ctx *c, const double *V, int nspin) { return set_vloc_common(c, V, nspin, false); }
extern "C" int pw_set_vloc_device(pw_ctx *c, const double *V, int nspin) { return set_vloc_common(c, V, nspin, true); }

int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out);

namespace {
// betaNL[ik] of nbeta columns: FP64 storage (allocated once), filled by `fill`
// on the context stream, then its FP32 copy and the split-BF16 operands
template <class Fill>
int set_beta(pw_ctx *c, int ik, int nbeta, Fill fill) {
    int s;
    if (c->nbeta != 0 && c->nbeta != nbeta) return fail(c, PW_ERR_ARG, "nbeta %d differs from %d", nbeta, c->nbeta);
    CK(c, cudaSetDevice(c->device));
    KData &kd = c->k[ik];
    const size_t n = (size_t)kd.Ngw * nbeta;
    if (!kd.d_beta64) {
        if ((s = dalloc(c, &kd.d_beta64, n)) || (s = dalloc(c, &kd.d_beta32, n))) return s;
    }
    if ((s = fill(kd.d_beta64))) return s;
    CK(c, convert_c128_to_c64(kd.d_beta64, kd.d_beta32, n, c->stream));
    if (c->use_umma) {
        // split-BF16 copies of betaNL for both tensor-core products, built once
        for (UmmaOperand *op : {&kd.beta_tn, &kd.beta_nn}) {
            const int64_t rows = (op == &kd.beta_tn) ? 2 * (int64_t)nbeta : 2 * (int64_t)kd.Ngw;
            const int64_t K = (op == &kd.beta_tn) ? kd.Ngw : nbeta;
            if (!op->hi) {
                const size_t half = umma_operand_bytes(rows, K) / 2;
                if ((s = dalloc(c, (unsigned char **)&op->hi, half)) || (s = dalloc(c, (unsigned char **)&op->lo, half)))
                    return s;
                // betaNL' psi runs with three pieces (see apply_T)
                if (op == &kd.beta_tn && (s = dalloc(c, (unsigned char **)&op->lo2, half))) return s;
            }
        }
        CK(c, umma_prep_tn_a<float2>(kd.d_beta32, kd.Ngw, kd.Ngw, nbeta, kd.beta_tn, c->stream));
        CK(c, umma_prep_nn_a<float2>(kd.d_beta32, kd.Ngw, kd.Ngw, nbeta, kd.beta_nn, c->stream));
    }
    CK(c, cudaStreamSynchronize(c->stream));
    c->nbeta = nbeta;
    return PW_OK;
}
}  // namespace

extern "C" int pw_set_nonlocal(pw_ctx *c, int ik, const double *beta, int nbeta) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik))) return s;
    if (!beta || nbeta <= 0) return fail(c, PW_ERR_ARG, "empty betaNL");
    const size_t n = (size_t)c->k[ik].Ngw * nbeta;
    return set_beta(c, ik, nbeta, [&](double2 *d) {
        CK(c, cudaMemcpyAsync(d, beta, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        return (int)PW_OK;
    });
}

extern "C" int pw_build_nonlocal(pw_ctx *c, int ik, int nbeta, const int32_t *atom, const int32_t *l, const int32_t *m,
                                 const int32_t *iproj, const double *rc, const double *pref, int natoms,
                                 const double *pos) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik))) return s;
    if (nbeta <= 0 || natoms <= 0 || !atom || !l || !m || !iproj || !rc || !pref || !pos)
        return fail(c, PW_ERR_ARG, "bad projector table");
    if (!c->k[ik].d_gk) return fail(c, PW_ERR_STATE, "G+k vectors of k-point %d are not set (pw_set_gkvec)", ik);
    std::vector<ProjCol> cols(nbeta);
    for (int j = 0; j < nbeta; ++j) {
        const bool ok = atom[j] >= 0 && atom[j] < natoms && l[j] >= 0 && l[j] <= 3 && m[j] >= -l[j] && m[j] <= l[j] &&
                        iproj[j] >= 1 && iproj[j] <= (l[j] == 0 ? 3 : l[j] == 1 ? 3 : l[j] == 2 ? 2 : 1);
        if (!ok) return fail(c, PW_ERR_ARG, "projector column %d: unsupported (atom, l, m, i)", j);
        cols[j] = ProjCol{atom[j], l[j], m[j], iproj[j], rc[j], pref[j]};
    }
    CK(c, cudaSetDevice(c->device));
    ProjCol *d_cols = nullptr;
    double *d_pos = nullptr;
    if ((s = pwk_scratch(c, SL_FRC_A, nbeta * sizeof(ProjCol), (void **)&d_cols)) ||
        (s = pwk_scratch(c, SL_FRC_B, 3 * (size_t)natoms * sizeof(double), (void **)&d_pos)))
        return s;
    CK(c, cudaMemcpyAsync(d_cols, cols.data(), nbeta * sizeof(ProjCol), cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(d_pos, pos, 3 * (size_t)natoms * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const KData &kd = c->k[ik];
    return set_beta(c, ik, nbeta, [&](double2 *d) {
        CK(c, launch_build_beta(kd.d_gk, kd.Ngw, d_cols, nbeta, d_pos, d, c->stream));
        c->launches += 1;
        return (int)PW_OK;
    });
}

extern "C" int pw_set_nonlocal_coef(pw_ctx *c, int nnz, const int32_t *ib, const int32_t *jb, const double *h) {
    if (!c) return PW_ERR_ARG;
    if (c->nbeta <= 0) return fail(c, PW_ERR_STATE, "call pw_set_nonlocal before pw_set_nonlocal_coef");
    if (nnz < 0 || (nnz > 0 && (!ib || !jb || !h))) return fail(c, PW_ERR_ARG, "invalid coefficient list");
    std::vector<std::vector<std::pair<int, double>>> rows(c->nbeta);
    for (int e = 0; e < nnz; ++e) {
        if (ib[e] < 0 || ib[e] >= c->nbeta || jb[e] < 0 || jb[e] >= c->nbeta)
            return fail(c, PW_ERR_ARG, "coefficient %d: index outside [0, %d)", e, c->nbeta);
        bool merged = false;
        for (auto &pr : rows[ib[e]])
            if (pr.first == jb[e]) {
                pr.second += h[e];
                merged = true;
            }
        if (!merged) rows[ib[e]].push_back({jb[e], h[e]});
    }
    std::vector<int> rp(c->nbeta + 1, 0), col;
    std::vector<double> val;
    for (int i = 0; i < c->nbeta; ++i) {
        for (auto &pr : rows[i]) {
            col.push_back(pr.first);
            val.push_back(pr.second);
        }
        rp[i + 1] = (int)col.size();
    }
    CK(c, cudaSetDevice(c->device));
    dfree(c, c->d_Drow);
    dfree(c, c->d_Dcol);
    dfree(c, c->d_Dval);
    int s;
    if ((s = upload(c, &c->d_Drow, rp)) || (s = upload(c, &c->d_Dcol, col)) || (s = upload(c, &c->d_Dval, val))) return s;
    c->have_D = true;
    return PW_OK;
}

extern "C" int pw_apply(pw_ctx *c, int ik, int ispin, int dtype, const void *psi, void *Hpsi, int64_t ld, int nb,
                        unsigned ops) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!psi || !Hpsi) return fail(c, PW_ERR_ARG, "NULL wavefunction pointer");
    if (psi == Hpsi) return fail(c, PW_ERR_ARG, "psi and Hpsi must not alias");
    if (nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad shape: nb=%d ld=%lld Ngw=%d", nb, (long long)ld, c->k[ik].Ngw);
    if (ops & ~(PW_OP_H | PW_ACCUMULATE)) return fail(c, PW_ERR_ARG, "unknown op flags 0x%x", ops);
    CK(c, cudaSetDevice(c->device));
    return dtype == PW_C128 ? apply_T<double>(c, ik, ispin, psi, Hpsi, ld, nb, ops)
                            : apply_T<float>(c, ik, ispin, psi, Hpsi, ld, nb, ops);
}

// ------------------------------------------------- batched op_H (k-points)
namespace {
uint64_t fnv(uint64_t h, const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

template <typename T>
int apply_multi_T(pw_ctx *c, int nk, const int *iks, int ispin, void *const *psi, void *const *Hpsi, const int64_t *ld,
                  const int *nb, unsigned ops) {
    const unsigned o = ops & PW_OP_H;
    const size_t es = 2 * sizeof(T);
    if (!(o & PW_OP_VLOC)) return fail(c, PW_ERR_UNSUPPORTED, "the batched op_H needs PW_OP_VLOC");
    if (c->N1 != c->N2 || c->N2 != c->N3 || (c->N1 != 27 && c->N1 != 75 && c->N1 != 120))
        return fail(c, PW_ERR_UNSUPPORTED, "the batched op_H runs on cube grids of 27, 75 or 120 points");
    if (c->vloc_nspin <= 0) return fail(c, PW_ERR_STATE, "op_V_loc requested before pw_set_vloc");
    if (ispin < 0 || ispin >= c->vloc_nspin) return fail(c, PW_ERR_ARG, "spin index %d outside [0, %d)", ispin, c->vloc_nspin);
    const bool vnl = (o & PW_OP_VNL) != 0;
    if (vnl && (c->nbeta <= 0 || !c->have_D)) return fail(c, PW_ERR_STATE, "op_V_Ps_nloc requested but projectors are not set");
    if (vnl && c->nbeta > 2048) return fail(c, PW_ERR_UNSUPPORTED, "the batched op_V_Ps_nloc takes at most 2048 projectors");
    std::vector<MkK> tab(nk);
    std::vector<int> band_k;
    size_t aoff = 0;
    int maxcol = 0, maxnb = 0, kx = iks[0];
    for (int i = 0; i < nk; ++i) {
        const KData &kd = c->k[iks[i]];
        const void *beta = sizeof(T) == 8 ? (const void *)kd.d_beta64 : (const void *)kd.d_beta32;
        if (vnl && !beta) return fail(c, PW_ERR_STATE, "projectors of k-point %d are not set", iks[i]);
        MkK &K = tab[i];
        K.kp = make_launch<T>(c, iks[i]).kp;
        K.psi = psi[i];
        K.Hpsi = Hpsi[i];
        K.beta = vnl ? beta : nullptr;
        K.ld = ld[i];
        K.a_off = aoff;
        K.band0 = (int)band_k.size();
        K.nb = nb[i];
        aoff += (size_t)nb[i] * c->N3 * kd.Ncol;
        band_k.insert(band_k.end(), nb[i], i);
        maxcol = std::max(maxcol, kd.Ncol);
        maxnb = std::max(maxnb, nb[i]);
        if (kd.Nxa > c->k[kx].Nxa) kx = iks[i];
    }
    const int nbands = (int)band_k.size();
    if (nbands > 65535) return fail(c, PW_ERR_UNSUPPORTED, "the batched op_H takes at most 65535 bands per call");
    int s;
    if ((s = ensure(c, c->A, aoff * es))) return s;
    const size_t tab_bytes = (size_t)nk * sizeof(MkK), bk_bytes = (size_t)nbands * sizeof(int);
    const size_t bk_off = (tab_bytes + 255) / 256 * 256;
    const size_t ctr_off = (bk_off + bk_bytes + 255) / 256 * 256;   // grid-barrier counter of the persistent launch
    if ((s = ensure(c, c->mk_tab, ctr_off + 256))) return s;
    const void *V = sizeof(T) == 8 ? (const void *)(c->d_V64 + (size_t)ispin * c->N)
                                   : (const void *)(c->d_V32 + (size_t)ispin * c->N);
    const int flags = ((o & PW_OP_K) ? 2 : 0) | ((ops & PW_ACCUMULATE) ? 4 : 0);
    const FftLaunch L = make_launch<T>(c, kx);
    const MkK *d_tab = (const MkK *)c->mk_tab.p;
    const int *d_bk = (const int *)((const char *)c->mk_tab.p + bk_off);
    unsigned *d_ctr = (unsigned *)((char *)c->mk_tab.p + ctr_off);
    // graph replay: same blocks, k-points, flags and buffers as the captured call
    uint64_t key = 1469598103934665603ull;
    key = fnv(key, tab.data(), tab_bytes);
    key = fnv(key, &V, sizeof(V));
    key = fnv(key, &c->A.p, sizeof(void *));
    key = fnv(key, &c->mk_tab.p, sizeof(void *));
    key = fnv(key, &flags, sizeof(flags));
    const unsigned pflag = ops & PW_PERSISTENT;
    key = fnv(key, &pflag, sizeof(pflag));
    key = fnv(key, &nbands, sizeof(nbands));
    if ((ops & PW_GRAPH) && c->mk_exec && key == c->mk_key) {
        CK(c, cudaGraphLaunch(c->mk_exec, c->stream));
        c->launches += c->mk_nlaunch;
        return PW_OK;
    }
    CK(c, cudaMemcpyAsync(c->mk_tab.p, tab.data(), tab_bytes, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync((char *)c->mk_tab.p + bk_off, band_k.data(), bk_bytes, cudaMemcpyHostToDevice, c->stream));
    // one persistent cooperative launch for every stage (the per-stage
    // launches when it does not fit or a stream capture refuses it)
    bool persistent = (ops & PW_PERSISTENT) != 0;
    int nlaunch = 1;
    auto run = [&](cudaStream_t st) {
        if (persistent) {
            const cudaError_t e = launch_multik_persistent<T>(L, d_tab, d_bk, nbands, maxcol, V, c->A.p, flags,
                                                              c->d_Drow, c->d_Dcol, c->d_Dval, vnl ? c->nbeta : 0,
                                                              d_ctr, c->d_err, st);
            if (e == cudaSuccess) {
                nlaunch = 1;
                return e;
            }
            if (e != cudaErrorCooperativeLaunchTooLarge && e != cudaErrorNotSupported) return e;
            persistent = false;
        }
        nlaunch = vnl ? 4 : 3;
        return launch_multik<T>(L, d_tab, d_bk, nk, nbands, maxnb, maxcol, V, c->A.p, flags, c->d_Drow, c->d_Dcol,
                                c->d_Dval, vnl ? c->nbeta : 0, st);
    };
    CK(c, run(c->stream));
    c->launches += nlaunch;
    if (ops & PW_GRAPH) {
        // capture the same launches for replay (the tables stay resident)
        CK(c, cudaStreamSynchronize(c->stream));
        if (!c->cap_stream) CK(c, cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
        if (c->mk_exec) {
            CK(c, cudaGraphExecDestroy(c->mk_exec));
            c->mk_exec = nullptr;
            c->mk_key = 0;
        }
        cudaGraph_t g = nullptr;
        CK(c, cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeRelaxed));
        cudaError_t e = run(c->cap_stream);
        cudaError_t e2 = cudaStreamEndCapture(c->cap_stream, &g);
        if ((e != cudaSuccess || e2 != cudaSuccess) && persistent) {
            // the capture refused the cooperative launch: capture the per-stage launches
            if (g) cudaGraphDestroy(g);
            g = nullptr;
            cudaGetLastError();
            persistent = false;
            CK(c, cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeRelaxed));
            e = run(c->cap_stream);
            e2 = cudaStreamEndCapture(c->cap_stream, &g);
        }
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(c, PW_ERR_CUDA, "capturing the batched op_H failed: %s",
                        cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        const cudaError_t e3 = cudaGraphInstantiate(&c->mk_exec, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            c->mk_exec = nullptr;
            return fail(c, PW_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e3));
        }
        c->mk_key = key;
        c->mk_nlaunch = nlaunch;
    }
    return PW_OK;
}
}  // namespace

extern "C" int pw_apply_multi(pw_ctx *c, int nk, const int *iks, int ispin, int dtype, void *const *psi,
                              void *const *Hpsi, const int64_t *ld, const int *nb, unsigned ops) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_dtype(c, dtype))) return s;
    if (nk <= 0 || !iks || !psi || !Hpsi || !ld || !nb) return fail(c, PW_ERR_ARG, "bad pw_apply_multi arguments");
    if (ops & ~(PW_OP_H | PW_ACCUMULATE | PW_GRAPH | PW_PERSISTENT)) return fail(c, PW_ERR_ARG, "unknown op flags 0x%x", ops);
    for (int i = 0; i < nk; ++i) {
        if ((s = check_k(c, iks[i]))) return s;
        if (!psi[i] || !Hpsi[i]) return fail(c, PW_ERR_ARG, "NULL wavefunction pointer (entry %d)", i);
        if (psi[i] == Hpsi[i]) return fail(c, PW_ERR_ARG, "psi and Hpsi must not alias (entry %d)", i);
        if (nb[i] <= 0 || ld[i] < c->k[iks[i]].Ngw) return fail(c, PW_ERR_ARG, "bad shape of entry %d", i);
    }
    CK(c, cudaSetDevice(c->device));
    return dtype == PW_C128 ? apply_multi_T<double>(c, nk, iks, ispin, psi, Hpsi, ld, nb, ops)
                            : apply_multi_T<float>(c, nk, iks, ispin, psi, Hpsi, ld, nb, ops);
}

extern "C" int pw_kprec(pw_ctx *c, int ik, int dtype, const void *in, void *out, int64_t ld, int nb) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!in || !out || nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad Kprec arguments");
    CK(c, cudaSetDevice(c->device));
    const KData &kd = c->k[ik];
    if (dtype == PW_C128)
        CK(c, launch_kprec<double>(kd.Ngw, nb, kd.d_Gk2, in, out, ld, c->stream));
    else
        CK(c, launch_kprec<float>(kd.Ngw, nb, kd.d_Gk2, in, out, ld, c->stream));
    return PW_OK;
}

extern "C" int pw_calc_rhoe(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, const double *w,
                            double *rhoe, int accumulate) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!psi || !w || !rhoe || nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad calc_rhoe arguments");
    CK(c, cudaSetDevice(c->device));
    return dtype == PW_C128 ? rhoe_T<double>(c, ik, psi, ld, nb, w, rhoe, accumulate)
                            : rhoe_T<float>(c, ik, psi, ld, nb, w, rhoe, accumulate);
}

// Adjoint of op_V_loc with respect to V: dV (+)= sum_b w_b N Re(conj(u_lam) u_psi)
// with u = G_to_R(.).  The density kernels give sum_b (w'_b / Omega) |N u_b|^2,
// so w' = w Omega / N; for lam != psi the polarised block [psi + lam, psi - lam]
// goes through them with weights +-w'/4.
template <typename T>
int vjp_T(pw_ctx *c, int ik, const void *psi, const void *lam, int64_t ld, int nb, const double *w, double *dV,
          int accumulate) {
    const double scale = c->CellVolume / (double)c->N;
    if (!lam || lam == psi) {
        std::vector<double> wv(w, w + nb);
        for (auto &x : wv) x *= scale;
        return rhoe_T<T>(c, ik, psi, ld, nb, wv.data(), dV, accumulate);
    }
    const KData &kd = c->k[ik];
    const size_t es = 2 * sizeof(T);
    int s;
    if ((s = ensure(c, c->slots[SL_VJP], 2 * (size_t)nb * kd.Ngw * es))) return s;
    CK(c, launch_polarize<T>(kd.Ngw, nb, psi, lam, ld, c->slots[SL_VJP].p, c->stream));
    c->launches += 1;
    std::vector<double> wv(2 * (size_t)nb);
    for (int b = 0; b < nb; ++b) {
        wv[b] = 0.25 * w[b] * scale;
        wv[nb + b] = -0.25 * w[b] * scale;
    }
    return rhoe_T<T>(c, ik, c->slots[SL_VJP].p, kd.Ngw, 2 * nb, wv.data(), dV, accumulate);
}

extern "C" int pw_vloc_vjp(pw_ctx *c, int ik, int dtype, const void *psi, const void *lam, int64_t ld, int nb,
                           const double *w, double *dV, int accumulate) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!psi || !w || !dV || nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad pw_vloc_vjp arguments");
    if (2 * (int64_t)nb > 65535 * 8) return fail(c, PW_ERR_ARG, "pw_vloc_vjp: nb too large");
    CK(c, cudaSetDevice(c->device));
    return dtype == PW_C128 ? vjp_T<double>(c, ik, psi, lam, ld, nb, w, dV, accumulate)
                            : vjp_T<float>(c, ik, psi, lam, ld, nb, w, dV, accumulate);
}

extern "C" int pw_gram(pw_ctx *c, int dtype, int64_t K, int m, int n, const void *A, int64_t lda, const void *B,
                       int64_t ldb, double *C, int64_t ldc, int accumulate) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_dtype(c, dtype))) return s;
    if (!A || !B || !C || K <= 0 || m <= 0 || n <= 0 || lda < K || ldb < K || ldc < m)
        return fail(c, PW_ERR_ARG, "bad gram arguments");
    CK(c, cudaSetDevice(c->device));
    if (dtype == PW_C64 && c->use_umma) return umma_tn<double2>(c, K, m, n, A, lda, B, ldb, C, ldc, accumulate);
    if ((s = ensure(c, c->gemm_ws, gemm_tn_ws_bytes(K, m, n)))) return s;
    if (dtype == PW_C128)
        CK(c, gemm_tn<double>(K, m, n, A, lda, B, ldb, (double2 *)C, ldc, accumulate, c->gemm_ws.p, c->stream));
    else
        CK(c, gemm_tn<float>(K, m, n, A, lda, B, ldb, (double2 *)C, ldc, accumulate, c->gemm_ws.p, c->stream));
    c->launches += 2;
    return PW_OK;
}

// Hermitian Gram (A^H B with the result known to be Hermitian, e.g. A = B
// or B = H A): only the upper triangle C[i][j], i <= j, is formed and
// written, in half the tiles.  Internal to the eigensolver paths, whose
// consumers read the upper triangle (Julia's Hermitian(.)).
int pwk_gram_upper(pw_ctx *c, int dtype, int64_t K, int m, const void *A, int64_t lda, const void *B, int64_t ldb,
                   double *C, int64_t ldc) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_dtype(c, dtype))) return s;
    if (!A || !B || !C || K <= 0 || m <= 0 || lda < K || ldb < K || ldc < m) return fail(c, PW_ERR_ARG, "bad gram arguments");
    CK(c, cudaSetDevice(c->device));
    if (dtype == PW_C64 && c->use_umma) return umma_tn<double2>(c, K, m, m, A, lda, B, ldb, C, ldc, 0, 1);
    if ((s = ensure(c, c->gemm_ws, gemm_tn_ws_bytes(K, m, m)))) return s;
    if (dtype == PW_C128)
        CK(c, gemm_tn<double>(K, m, m, A, lda, B, ldb, (double2 *)C, ldc, 0, c->gemm_ws.p, c->stream, 1));
    else
        CK(c, gemm_tn<float>(K, m, m, A, lda, B, ldb, (double2 *)C, ldc, 0, c->gemm_ws.p, c->stream, 1));
    c->launches += 2;
    return PW_OK;
}

extern "C" int pw_rotate(pw_ctx *c, int dtype, int64_t M, int n, int k, const void *A, int64_t lda, const double *U,
                         int64_t ldu, void *C, int64_t ldc, int accumulate) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_dtype(c, dtype))) return s;
    if (!A || !U || !C || M <= 0 || n <= 0 || k <= 0 || lda < M || ldu < k || ldc < M)
        return fail(c, PW_ERR_ARG, "bad rotate arguments");
    if (A == C) return fail(c, PW_ERR_ARG, "A and C must not alias");
    CK(c, cudaSetDevice(c->device));
    if (dtype == PW_C64 && c->use_umma)
        return umma_nn(c, M, n, k, A, lda, nullptr, (const double2 *)U, ldu, C, ldc, accumulate);
    if (dtype == PW_C128)
        CK(c, gemm_nn<double>(M, n, k, A, lda, (const double2 *)U, ldu, C, ldc, accumulate, c->stream));
    else
        CK(c, gemm_nn<float>(M, n, k, A, lda, (const double2 *)U, ldu, C, ldc, accumulate, c->stream));
    c->launches += 1;
    return PW_OK;
}

extern "C" int pw_op_H_host(pw_ctx *c, int ik, int ispin, const double *psi, double *Hpsi, int64_t ld, int nb,
                            unsigned ops, int dtype) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!psi || !Hpsi || nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad op_H arguments");
    CK(c, cudaSetDevice(c->device));
    const size_t n = (size_t)ld * nb;
    const bool acc = (ops & PW_ACCUMULATE) != 0;
    if ((s = ensure(c, c->st_in, n * sizeof(double2))) || (s = ensure(c, c->st_out, n * sizeof(double2)))) return s;
    if (dtype == PW_C64 && ((s = ensure(c, c->st_in32, n * sizeof(float2))) || (s = ensure(c, c->st_out32, n * sizeof(float2)))))
        return s;
    // Pipelined over band chunks: the host-to-device copy of chunk i+1 and the
    // device-to-host copy of chunk i-1 run on their own streams while chunk i
    // computes on the context stream (each chunk has its own slice of the
    // staging buffers, so no slice is reused within a call).  Equal chunks of
    // about 32 bands (a ramp of small first and last chunks measured no gain
    // for the mixed path and 14 % slower for FP64, whose op_H outweighs the
    // copies).
    const int nch = std::max(1, std::min(8, nb / 32));
    const int cb = (nb + nch - 1) / nch;
    if (!c->cp_in) {
        CK(c, cudaStreamCreateWithFlags(&c->cp_in, cudaStreamNonBlocking));
        CK(c, cudaStreamCreateWithFlags(&c->cp_out, cudaStreamNonBlocking));
        for (int i = 0; i < 8; ++i) {
            CK(c, cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming));
            CK(c, cudaEventCreateWithFlags(&c->ev_cmp[i], cudaEventDisableTiming));
        }
    }
    // the copy streams must not start before work already queued on the context stream
    CK(c, cudaEventRecord(c->ev_cmp[0], c->stream));
    CK(c, cudaStreamWaitEvent(c->cp_in, c->ev_cmp[0], 0));
    for (int i = 0; i * cb < nb; ++i) {
        const int b0 = i * cb, cnt = std::min(cb, nb - b0);
        const size_t off = (size_t)b0 * ld, m = (size_t)cnt * ld;
        double2 *in64 = (double2 *)c->st_in.p + off, *out64 = (double2 *)c->st_out.p + off;
        CK(c, cudaMemcpyAsync(in64, psi + 2 * off, m * sizeof(double2), cudaMemcpyHostToDevice, c->cp_in));
        if (acc) CK(c, cudaMemcpyAsync(out64, Hpsi + 2 * off, m * sizeof(double2), cudaMemcpyHostToDevice, c->cp_in));
        CK(c, cudaEventRecord(c->ev_in[i], c->cp_in));
        CK(c, cudaStreamWaitEvent(c->stream, c->ev_in[i], 0));
        if (dtype == PW_C128) {
            if ((s = apply_T<double>(c, ik, ispin, in64, out64, ld, cnt, ops))) return s;
        } else {
            float2 *in32 = (float2 *)c->st_in32.p + off, *out32 = (float2 *)c->st_out32.p + off;
            CK(c, convert_c128_to_c64(in64, in32, m, c->stream));
            if (acc) CK(c, convert_c128_to_c64(out64, out32, m, c->stream));
            if ((s = apply_T<float>(c, ik, ispin, in32, out32, ld, cnt, ops))) return s;
            CK(c, convert_c64_to_c128(out32, out64, m, c->stream));
        }
        CK(c, cudaEventRecord(c->ev_cmp[i], c->stream));
        CK(c, cudaStreamWaitEvent(c->cp_out, c->ev_cmp[i], 0));
        CK(c, cudaMemcpyAsync(Hpsi + 2 * off, out64, m * sizeof(double2), cudaMemcpyDeviceToHost, c->cp_out));
    }
    CK(c, cudaStreamSynchronize(c->cp_out));
    CK(c, cudaStreamSynchronize(c->stream));
    return PW_OK;
}

extern "C" int pw_calc_rhoe_host(pw_ctx *c, int ik, const double *psi, int64_t ld, int nb, const double *w,
                                 double *rhoe, int accumulate, int dtype) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (!psi || !w || !rhoe || nb <= 0 || ld < c->k[ik].Ngw) return fail(c, PW_ERR_ARG, "bad calc_rhoe arguments");
    CK(c, cudaSetDevice(c->device));
    const size_t n = (size_t)ld * nb;
    if ((s = ensure(c, c->st_in, n * sizeof(double2))) || (s = ensure(c, c->st_rho, c->N * sizeof(double)))) return s;
    CK(c, cudaMemcpyAsync(c->st_in.p, psi, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    if (accumulate) CK(c, cudaMemcpyAsync(c->st_rho.p, rhoe, c->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (dtype == PW_C128) {
        if ((s = rhoe_T<double>(c, ik, c->st_in.p, ld, nb, w, (double *)c->st_rho.p, accumulate))) return s;
    } else {
        if ((s = ensure(c, c->st_in32, n * sizeof(float2)))) return s;
        CK(c, convert_c128_to_c64((const double2 *)c->st_in.p, (float2 *)c->st_in32.p, n, c->stream));
        if ((s = rhoe_T<float>(c, ik, c->st_in32.p, ld, nb, w, (double *)c->st_rho.p, accumulate))) return s;
    }
    CK(c, cudaMemcpyAsync(rhoe, c->st_rho.p, c->N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return PW_OK;
}

// ------------------------------------------------------------------------
// Internal accessors used by the allocation-free entry point (pw_noalloc.cu).
int pwk_fail(pw_ctx *c, int code, const char *msg) { return fail(c, code, "%s", msg); }

void pwk_count_launches(pw_ctx *c, int n) { c->launches += n; }

// Validates (ik, ispin, dtype) for an op_V_loc round trip and returns the
// launch description, the V(r)/N pointer of the precision, the stream, the
// scratch bytes one band needs, and the context's device.  Allocates nothing.
int pwk_vloc_view(pw_ctx *c, int ik, int ispin, int dtype, pwk::FftLaunch *L, const void **V, cudaStream_t *st,
                  size_t *per_band, int *device) {
    int s;
    if ((s = check_k(c, ik)) || (s = check_dtype(c, dtype))) return s;
    if (c->vloc_nspin <= 0) return fail(c, PW_ERR_STATE, "op_V_loc requested before pw_set_vloc");
    if (ispin < 0 || ispin >= c->vloc_nspin) return fail(c, PW_ERR_ARG, "spin index %d outside [0, %d)", ispin, c->vloc_nspin);
    const bool dbl = dtype == PW_C128;
    *L = dbl ? make_launch<double>(c, ik) : make_launch<float>(c, ik);
    *V = dbl ? (const void *)(c->d_V64 + (size_t)ispin * c->N) : (const void *)(c->d_V32 + (size_t)ispin * c->N);
    *st = c->stream;
    *per_band = (size_t)c->N3 * c->k[ik].Ncol * (dbl ? sizeof(double2) : sizeof(float2));
    *device = c->device;
    return PW_OK;
}

int pwk_ngw(const pw_ctx *c, int ik) { return c->k[ik].Ngw; }

// Shape of k-point ik for the autotuner's cache key.
int pwk_tune_shape(const pw_ctx *c, int ik, int *Ns, int *Ncol, int *Nxa, int *nbeta) {
    if (ik < 0 || ik >= c->Nkpt) return PW_ERR_ARG;
    Ns[0] = c->N1;
    Ns[1] = c->N2;
    Ns[2] = c->N3;
    *Ncol = c->k[ik].Ncol;
    *Nxa = c->k[ik].Nxa;
    *nbeta = (c->nbeta > 0 && c->have_D) ? c->nbeta : 0;
    return PW_OK;
}
int pwk_fail_msg(pw_ctx *c, int code, const char *msg) { return fail(c, code, "%s", msg); }
void **pwk_mix_slot(pw_ctx *c) { return &c->mix_state; }

int pwk_scratch(pw_ctx *c, int slot, size_t bytes, void **out) {
    if (slot < 0 || slot >= 32) return fail(c, PW_ERR_ARG, "scratch slot %d", slot);
    int s = ensure(c, c->slots[slot], bytes);
    if (s) return s;
    *out = c->slots[slot].p;
    return PW_OK;
}
cudaStream_t pwk_stream(pw_ctx *c) { return c->stream; }
int pwk_device(const pw_ctx *c) { return c->device; }
int pwk_nkpt(const pw_ctx *c) { return c->Nkpt; }

int pwk_density_launch(pw_ctx *c, pwk::FftLaunch *L, const double **G2, int *Ng, size_t *N) {
    if (!c->have_dens) return fail(c, PW_ERR_STATE, "call pw_set_density_sphere first");
    *L = make_launch_kd<double>(c, c->dens);
    *G2 = c->dens.d_Gk2;
    *Ng = c->dens.Ngw;
    *N = c->N;
    return PW_OK;
}
int pwk_set_vloc_device(pw_ctx *c, const double *V, int nspin) { return set_vloc_common(c, V, nspin, true); }
const double *pwk_gk2(const pw_ctx *c, int ik) { return c->k[ik].d_Gk2; }

// out (nbeta x nb, FP64 complex) = betaNL' psi for k-point ik (betaNL' psi
// with three BF16 pieces on the mixed path, as in op_H)
int pwk_beta_dot(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, double2 *out) {
    const KData &kd = c->k[ik];
    const void *beta = dtype == PW_C128 ? (const void *)kd.d_beta64 : (const void *)kd.d_beta32;
    if (c->nbeta <= 0 || !beta) return fail(c, PW_ERR_STATE, "projectors of k-point %d are not set", ik);
    int s;
    cudaStream_t st = c->stream;
    if (dtype == PW_C64 && c->use_umma) {
        UmmaOperand B;
        if ((s = umma_scratch(c, c->um_b_hi, c->um_b_lo, nb, kd.Ngw, B, &c->um_b_lo2))) return s;
        CK(c, umma_prep_tn_b<float2>(psi, ld, kd.Ngw, nb, B, st));
        if ((s = ensure(c, c->um_ws, umma_ws_bytes(kd.beta_tn.rows, nb, kd.beta_tn.Kp)))) return s;
        CK(c, umma_gemm<double2>(kd.beta_tn, B, c->nbeta, nb, out, c->nbeta, 0, (float *)c->um_ws.p, c->d_err, st));
        c->launches += 2 + (umma_splits(kd.beta_tn.rows, nb, kd.beta_tn.Kp) > 1 ? 1 : 0);
    } else {
        if ((s = ensure(c, c->gemm_ws, gemm_tn_ws_bytes(kd.Ngw, c->nbeta, nb)))) return s;
        if (dtype == PW_C128)
            CK(c, (gemm_tn<double>(kd.Ngw, c->nbeta, nb, beta, kd.Ngw, psi, ld, out, c->nbeta, 0, c->gemm_ws.p, st)));
        else
            CK(c, (gemm_tn<float>(kd.Ngw, c->nbeta, nb, beta, kd.Ngw, psi, ld, out, c->nbeta, 0, c->gemm_ws.p, st)));
        c->launches += 2;
    }
    return PW_OK;
}

// P = betaNL' psi and P2 = D P for k-point ik into the context's buffers
int pwk_projections(pw_ctx *c, int ik, int dtype, const void *psi, int64_t ld, int nb, const double2 **P,
                    const double2 **P2, int *nbeta) {
    *nbeta = c->nbeta;
    if (c->nbeta <= 0) return PW_OK;
    if (!c->have_D) return fail(c, PW_ERR_STATE, "nonlocal coefficients are not set");
    int s;
    const size_t pb = (size_t)c->nbeta * nb * sizeof(double2);
    if ((s = ensure(c, c->P, pb)) || (s = ensure(c, c->P2, pb))) return s;
    cudaStream_t st = c->stream;
    if ((s = pwk_beta_dot(c, ik, dtype, psi, ld, nb, (double2 *)c->P.p))) return s;
    CK(c, apply_dcsr(c->nbeta, nb, c->d_Drow, c->d_Dcol, c->d_Dval, (const double2 *)c->P.p, (double2 *)c->P2.p, st));
    c->launches += 1;
    *P = (const double2 *)c->P.p;
    *P2 = (const double2 *)c->P2.p;
    return PW_OK;
}

extern "C" int pw_set_density_sphere(pw_ctx *c, int64_t Ng, const int64_t *idx_g2r, const double *G2, int index_base) {
    if (!c) return PW_ERR_ARG;
    if (!idx_g2r || !G2 || Ng <= 0 || (index_base != 0 && index_base != 1))
        return fail(c, PW_ERR_ARG, "bad density sphere");
    CK(c, cudaSetDevice(c->device));
    if (c->have_dens) return fail(c, PW_ERR_STATE, "density sphere already set");
    int s = build_kdata(c, c->dens, Ng, idx_g2r, index_base, G2);
    if (s) return s;
    c->have_dens = true;
    return PW_OK;
}

extern "C" int pw_set_xc(pw_ctx *c, int xc, const double *G) {
    if (!c) return PW_ERR_ARG;
    if (xc != PW_XC_VWN && xc != PW_XC_PBE) return fail(c, PW_ERR_ARG, "unknown exchange-correlation %d", xc);
    CK(c, cudaSetDevice(c->device));
    if (xc == PW_XC_PBE) {
        if (!c->have_dens) return fail(c, PW_ERR_STATE, "call pw_set_density_sphere before pw_set_xc(PBE)");
        if (!G) return fail(c, PW_ERR_ARG, "PBE needs the G vectors of the density sphere");
        const size_t ng = (size_t)c->dens.Ngw;
        int s;
        if (!c->d_xcG && (s = dalloc(c, &c->d_xcG, 3 * ng))) return s;
        CK(c, cudaMemcpy(c->d_xcG, G, 3 * ng * sizeof(double), cudaMemcpyHostToDevice));
    }
    c->xc = xc;
    return PW_OK;
}
extern "C" int pw_set_symmetry(pw_ctx *c, int nshell, int nsym, const int32_t *isg, const double *phase) {
    if (!c) return PW_ERR_ARG;
    if (!c->have_dens) return fail(c, PW_ERR_STATE, "call pw_set_density_sphere before pw_set_symmetry");
    if (nshell <= 0 || nsym <= 0 || !isg || !phase) return fail(c, PW_ERR_ARG, "bad symmetry tables");
    const size_t n = (size_t)nshell * nsym;
    for (size_t i = 0; i < n; ++i)
        if (isg[i] < 0 || isg[i] >= c->dens.Ngw) return fail(c, PW_ERR_ARG, "symmetry table index %d outside the sphere", isg[i]);
    CK(c, cudaSetDevice(c->device));
    dfree(c, c->d_sym_isg);
    dfree(c, c->d_sym_ph);
    c->d_sym_isg = nullptr;
    c->d_sym_ph = nullptr;
    int s;
    if ((s = dalloc(c, &c->d_sym_isg, n)) || (s = dalloc(c, &c->d_sym_ph, n))) return s;
    CK(c, cudaMemcpy(c->d_sym_isg, isg, n * sizeof(int), cudaMemcpyHostToDevice));
    CK(c, cudaMemcpy(c->d_sym_ph, phase, n * sizeof(double2), cudaMemcpyHostToDevice));
    c->sym_nshell = nshell;
    c->sym_nsym = nsym;
    return PW_OK;
}
int pwk_symmetry(const pw_ctx *c, const int **isg, const double2 **ph, int *nshell, int *nsym) {
    *isg = c->d_sym_isg;
    *ph = c->d_sym_ph;
    *nshell = c->sym_nshell;
    *nsym = c->sym_nsym;
    return c->d_sym_isg ? PW_OK : PW_ERR_STATE;
}
int pwk_xc(const pw_ctx *c, const double **G) {
    *G = c->d_xcG;
    return c->xc;
}

// ------------------------------------------------------------------ forces
extern "C" int pw_set_force_tables(pw_ctx *c, int nspecies, const double *VlocG, const double *G) {
    if (!c) return PW_ERR_ARG;
    if (!c->have_dens) return fail(c, PW_ERR_STATE, "call pw_set_density_sphere before pw_set_force_tables");
    if (nspecies <= 0 || !VlocG || !G) return fail(c, PW_ERR_ARG, "bad force tables");
    CK(c, cudaSetDevice(c->device));
    const size_t ng = (size_t)c->dens.Ngw;
    dfree(c, c->d_fG);
    dfree(c, c->d_fV);
    c->d_fG = nullptr;
    c->d_fV = nullptr;
    int s;
    if ((s = dalloc(c, &c->d_fG, 3 * ng)) || (s = dalloc(c, &c->d_fV, ng * nspecies))) return s;
    CK(c, cudaMemcpy(c->d_fG, G, 3 * ng * sizeof(double), cudaMemcpyHostToDevice));
    CK(c, cudaMemcpy(c->d_fV, VlocG, ng * nspecies * sizeof(double), cudaMemcpyHostToDevice));
    c->f_nsp = nspecies;
    return PW_OK;
}

extern "C" int pw_set_gkvec(pw_ctx *c, int ik, const double *gk) {
    if (!c) return PW_ERR_ARG;
    int s;
    if ((s = check_k(c, ik))) return s;
    if (!gk) return fail(c, PW_ERR_ARG, "NULL G+k vectors");
    CK(c, cudaSetDevice(c->device));
    KData &kd = c->k[ik];
    if (!kd.d_gk && (s = dalloc(c, &kd.d_gk, 3 * (size_t)kd.Ngw))) return s;
    CK(c, cudaMemcpy(kd.d_gk, gk, 3 * (size_t)kd.Ngw * sizeof(double), cudaMemcpyHostToDevice));
    return PW_OK;
}

extern "C" int pw_set_nonlocal_atoms(pw_ctx *c, int natoms, const int32_t *atom_of_beta) {
    if (!c) return PW_ERR_ARG;
    if (c->nbeta <= 0) return fail(c, PW_ERR_STATE, "call pw_set_nonlocal before pw_set_nonlocal_atoms");
    if (natoms <= 0 || !atom_of_beta) return fail(c, PW_ERR_ARG, "bad projector atom list");
    // the projectors of one atom are contiguous (PsPotNL.jl:147-195 order)
    std::vector<int> rows(natoms + 1, 0);
    int prev = -1;
    for (int b = 0; b < c->nbeta; ++b) {
        const int a = atom_of_beta[b];
        if (a < 0 || a >= natoms || a < prev) return fail(c, PW_ERR_ARG, "projector %d: atom %d out of order", b, a);
        for (int q = prev + 1; q <= a; ++q) rows[q] = b;
        prev = a;
    }
    for (int q = prev + 1; q <= natoms; ++q) rows[q] = c->nbeta;
    CK(c, cudaSetDevice(c->device));
    dfree(c, c->d_atom_rows);
    c->d_atom_rows = nullptr;
    int s;
    if ((s = upload(c, &c->d_atom_rows, rows))) return s;
    c->f_natoms = natoms;
    return PW_OK;
}

int pwk_force_local_tables(pw_ctx *c, const double **G, const double **V, int *nsp, int *ng) {
    if (!c->d_fG || !c->have_dens) return fail(c, PW_ERR_STATE, "force tables are not set (pw_set_force_tables)");
    *G = c->d_fG;
    *V = c->d_fV;
    *nsp = c->f_nsp;
    *ng = c->dens.Ngw;
    return PW_OK;
}
int pwk_force_nonlocal_tables(pw_ctx *c, int ik, const double **gk, const int **atom_rows, int *natoms, const int **rowptr,
                              const int **col, const double **val, int *nbeta) {
    if (!c->k[ik].d_gk) return fail(c, PW_ERR_STATE, "G+k vectors of k-point %d are not set (pw_set_gkvec)", ik);
    if (!c->d_atom_rows) return fail(c, PW_ERR_STATE, "projector atoms are not set (pw_set_nonlocal_atoms)");
    if (!c->have_D) return fail(c, PW_ERR_STATE, "nonlocal coefficients are not set");
    *gk = c->k[ik].d_gk;
    *atom_rows = c->d_atom_rows;
    *natoms = c->f_natoms;
    *rowptr = c->d_Drow;
    *col = c->d_Dcol;
    *val = c->d_Dval;
    *nbeta = c->nbeta;
    return PW_OK;
}
int pwk_grid_points(const pw_ctx *c, size_t *N) {
    *N = c->N;
    return PW_OK;
}
