// Pruned, band-batched 3-D FFT passes for op_V_loc! and calc_rhoe!.
//
// The reference does, per band, a dense scatter into an N-point grid, a full
// 3-D backward FFT, a pointwise product with V_loc, a full forward FFT and a
// gather (op_V_loc.jl:137-165).  Here the transform is split along its axes
// so that only non-zero data is ever transformed or stored:
//
//   K-zinv   per (band, column group): gather the sphere entries of each
//            active (x,y) column (those holding at least one G of the
//            wavefunction sphere), backward z-FFT, store A[b][z][col].
//   K-plane  per (band, z-plane): scatter the plane's Ncol column values into
//            an (active-x) x N2 sub-plane in SMEM, backward y-FFT on the
//            active-x lines, then for chunks of y lines expand to full x
//            lines, backward x-FFT, multiply by V(r)/N, forward x-FFT, keep
//            the active-x outputs; forward y-FFT; store the active columns
//            back to A.
//   K-zfwd   per (band, column group): forward z-FFT, gather the sphere
//            entries and write Hpsi = [Hpsi +] Vpsi [+ 0.5|G+k|^2 psi].
//   K-rho    per (band group, z-plane): as K-plane up to the backward x-FFT,
//            then rho_part += w_b |psi(r)|^2 / Omega.
//
// HBM traffic per band: psi once in, Hpsi once out, A (Ncol*N3 complex)
// written/read twice, V once per plane batch (L2-resident across bands).
#include <algorithm>

#include "pw_fft.cuh"
#include "pw_fft_tmpl.cuh"
#include "pw_fft_fused.cuh"

namespace pwk {

constexpr int FFT_THREADS = 256;

template <typename T> struct MaxV;
template <> struct MaxV<float> { static constexpr int v = 8; };
template <> struct MaxV<double> { static constexpr int v = 8; };

// ------------------------------------------------------------------ K-zinv
template <typename T>
__global__ void __launch_bounds__(FFT_THREADS, 2)
k_zinv(KPlan kp, FftDim dz, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ psi, int64_t ld,
       Cx<T> *__restrict__ A, int Cg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *tw = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *Z = tw + kp.N3;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * Cg;
    const int cn = min(Cg, kp.Ncol - c0);
    const int N3 = kp.N3;
    for (int i = threadIdx.x; i < N3; i += blockDim.x) tw[i] = twz[i];
    for (int i = threadIdx.x; i < N3 * Cg; i += blockDim.x) Z[i] = cmake((T)0, (T)0);
    __syncthreads();
    const int e0 = kp.col_ptr[c0], e1 = kp.col_ptr[c0 + cn];
    const Cx<T> *ps = psi + (size_t)b * ld;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int cl = kp.ent_col[e] - c0;
        Z[kp.ent_kz[e] * Cg + cl] = ps[kp.ent_igw[e]];
    }
    __syncthreads();
    fft_lines_w<T, MaxV<T>::v>(Z, dz, cn, Cg, 1, tw, +1);
    Cx<T> *Ab = A + (size_t)b * N3 * kp.Ncol;
    for (int p = threadIdx.x; p < N3 * cn; p += blockDim.x) {
        const int kz = p / cn, cl = p - kz * cn;
        Ab[(size_t)kz * kp.Ncol + c0 + cl] = Z[kz * Cg + cl];
    }
}

// ------------------------------------------------------------------ K-zfwd
// flags: 1 = add the V_loc part from A, 2 = add 0.5|G+k|^2 psi, 4 = accumulate into Hpsi
template <typename T>
__global__ void __launch_bounds__(FFT_THREADS, 2)
k_zfwd(KPlan kp, FftDim dz, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ A, const Cx<T> *__restrict__ psi,
       Cx<T> *__restrict__ Hpsi, int64_t ld, int Cg, int flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *tw = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *Z = tw + kp.N3;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * Cg;
    const int cn = min(Cg, kp.Ncol - c0);
    const int N3 = kp.N3;
    for (int i = threadIdx.x; i < N3; i += blockDim.x) tw[i] = twz[i];
    const Cx<T> *Ab = A + (size_t)b * N3 * kp.Ncol;
    for (int p = threadIdx.x; p < N3 * cn; p += blockDim.x) {
        const int kz = p / cn, cl = p - kz * cn;
        Z[kz * Cg + cl] = Ab[(size_t)kz * kp.Ncol + c0 + cl];
    }
    __syncthreads();
    fft_lines_w<T, MaxV<T>::v>(Z, dz, cn, Cg, 1, tw, -1);
    const int e0 = kp.col_ptr[c0], e1 = kp.col_ptr[c0 + cn];
    const Cx<T> *ps = psi + (size_t)b * ld;
    Cx<T> *hs = Hpsi + (size_t)b * ld;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int cl = kp.ent_col[e] - c0;
        const int igw = kp.ent_igw[e];
        Cx<T> out = Z[kp.ent_kz[e] * Cg + cl];
        if (flags & 2) {
            const T g2 = sizeof(T) == 8 ? (T)kp.ent_g2[e] : (T)kp.ent_g2f[e];
            out = cadd(out, cscale(ps[igw], (T)0.5 * g2));
        }
        if (flags & 4) out = cadd(out, hs[igw]);
        hs[igw] = out;
    }
}

// Shared-memory layout of the plane kernels.
struct PlaneSmem {
    int N1, N2, Nxa, Jc;
    __host__ __device__ size_t elems() const { return (size_t)N1 + N2 + (size_t)Nxa * N2 + (size_t)Jc * N1; }
};

// ----------------------------------------------------------------- K-plane
// Vr: V(r)/N for this spin channel, N1*N2*N3 reals, x fastest.
template <typename T>
__global__ void __launch_bounds__(FFT_THREADS, 2)
k_plane_vloc(KPlan kp, FftDim dx, FftDim dy, const Cx<T> *__restrict__ twx, const Cx<T> *__restrict__ twy,
             const T *__restrict__ Vr, Cx<T> *__restrict__ A, int Jc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = kp.N1, N2 = kp.N2, N3 = kp.N3, Nxa = kp.Nxa, Ncol = kp.Ncol;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N1;
    Cx<T> *S = ty + N2;               // [Nxa][N2]
    Cx<T> *X = S + (size_t)Nxa * N2;  // [Jc][N1]
    const int kz = blockIdx.x;
    const int b = blockIdx.y;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[i];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[i];
    for (int i = threadIdx.x; i < Nxa * N2; i += blockDim.x) S[i] = cmake((T)0, (T)0);
    __syncthreads();
    Cx<T> *Ap = A + ((size_t)b * N3 + kz) * Ncol;
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
    __syncthreads();
    fft_lines_w<T, MaxV<T>::v>(S, dy, Nxa, 1, N2, ty, +1);
    const T *Vp = Vr + (size_t)kz * N1 * N2;
    for (int j0 = 0; j0 < N2; j0 += Jc) {
        const int jc = min(Jc, N2 - j0);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = cmake((T)0, (T)0);
        __syncthreads();
        for (int p = threadIdx.x; p < Nxa * jc; p += blockDim.x) {
            const int ia = p / jc, jl = p - ia * jc;
            X[jl * N1 + kp.xa[ia]] = S[ia * N2 + j0 + jl];
        }
        __syncthreads();
        fft_lines_w<T, MaxV<T>::v>(X, dx, jc, 1, N1, tx, +1);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = cscale(X[i], Vp[(size_t)j0 * N1 + i]);
        __syncthreads();
        fft_lines_w<T, MaxV<T>::v>(X, dx, jc, 1, N1, tx, -1);
        for (int p = threadIdx.x; p < Nxa * jc; p += blockDim.x) {
            const int ia = p / jc, jl = p - ia * jc;
            S[ia * N2 + j0 + jl] = X[jl * N1 + kp.xa[ia]];
        }
        __syncthreads();
    }
    fft_lines_w<T, MaxV<T>::v>(S, dy, Nxa, 1, N2, ty, -1);
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) Ap[c] = S[kp.col_ia[c] * N2 + kp.col_j[c]];
}

// ------------------------------------------------------------------- K-rho
// rho_part[g][ip] (+)= sum over the group's bands of w_b |bfft psi_b(r)|^2
// (w_b already divided by Omega).  Each CTA owns plane kz of partial g.
template <typename T>
__global__ void __launch_bounds__(FFT_THREADS, 2)
k_plane_rho(KPlan kp, FftDim dx, FftDim dy, const Cx<T> *__restrict__ twx, const Cx<T> *__restrict__ twy,
            const Cx<T> *__restrict__ A, int nb, int Bg, const double *__restrict__ w, T *__restrict__ rho_part, int Jc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = kp.N1, N2 = kp.N2, N3 = kp.N3, Nxa = kp.Nxa, Ncol = kp.Ncol;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N1;
    Cx<T> *S = ty + N2;
    Cx<T> *X = S + (size_t)Nxa * N2;
    const int kz = blockIdx.x;
    const int g = blockIdx.y;
    const size_t N12 = (size_t)N1 * N2;
    T *rp = rho_part + (size_t)g * N12 * N3 + (size_t)kz * N12;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[i];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[i];
    for (size_t i = threadIdx.x; i < N12; i += blockDim.x) rp[i] = (T)0;
    const int b0 = g * Bg, b1 = min(nb, b0 + Bg);
    for (int b = b0; b < b1; ++b) {
        const T wb = (T)w[b];
        for (int i = threadIdx.x; i < Nxa * N2; i += blockDim.x) S[i] = cmake((T)0, (T)0);
        __syncthreads();
        const Cx<T> *Ap = A + ((size_t)b * N3 + kz) * Ncol;
        for (int c = threadIdx.x; c < Ncol; c += blockDim.x) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
        __syncthreads();
        fft_lines_w<T, MaxV<T>::v>(S, dy, Nxa, 1, N2, ty, +1);
        for (int j0 = 0; j0 < N2; j0 += Jc) {
            const int jc = min(Jc, N2 - j0);
            for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = cmake((T)0, (T)0);
            __syncthreads();
            for (int p = threadIdx.x; p < Nxa * jc; p += blockDim.x) {
                const int ia = p / jc, jl = p - ia * jc;
                X[jl * N1 + kp.xa[ia]] = S[ia * N2 + j0 + jl];
            }
            __syncthreads();
            fft_lines_w<T, MaxV<T>::v>(X, dx, jc, 1, N1, tx, +1);
            for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) {
                const Cx<T> v = X[i];
                rp[(size_t)j0 * N1 + i] += wb * (v.x * v.x + v.y * v.y);
            }
            __syncthreads();
        }
    }
}

// rho[ip] (+)= sum_g rho_part[g][ip]   (FP64 output)
template <typename T>
__global__ void k_rho_reduce(const T *__restrict__ part, int G, size_t N, double *__restrict__ rho, int accumulate) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        double s = accumulate ? rho[i] : 0.0;
        for (int g = 0; g < G; ++g) s += (double)part[(size_t)g * N + i];
        rho[i] = s;
    }
}

// --------------------------------------------------------- elementwise ops
// Hpsi (+)= 0.5 |G+k|^2 psi   (op_K.jl:67-73)
template <typename T>
__global__ void k_opK(int Ngw, int nb, const double *__restrict__ Gk2, const Cx<T> *__restrict__ psi,
                      Cx<T> *__restrict__ Hpsi, int64_t ld, int accumulate) {
    const size_t total = (size_t)Ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / Ngw), g = (int)(t - (size_t)b * Ngw);
        const size_t o = (size_t)b * ld + g;
        Cx<T> v = cscale(psi[o], (T)(0.5 * Gk2[g]));
        if (accumulate) v = cadd(v, Hpsi[o]);
        Hpsi[o] = v;
    }
}

// out = in / (1 + |G+k|^2)   (Kprec.jl:30-44)
template <typename T>
__global__ void k_kprec(int Ngw, int nb, const double *__restrict__ Gk2, const Cx<T> *in, Cx<T> *out, int64_t ld) {
    const size_t total = (size_t)Ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / Ngw), g = (int)(t - (size_t)b * Ngw);
        const size_t o = (size_t)b * ld + g;
        out[o] = cscale(in[o], (T)(1.0 / (1.0 + Gk2[g])));
    }
}

// out[b] = psi_b + lam_b, out[nb + b] = psi_b - lam_b (out: 2 nb columns of
// Ngw): the polarisation Re(conj(l) p) = (|p + l|^2 - |p - l|^2) / 4 that
// turns the density kernels into the adjoint of op_V_loc with respect to V
template <typename T>
__global__ void k_polarize(int Ngw, int nb, const Cx<T> *__restrict__ psi, const Cx<T> *__restrict__ lam, int64_t ld,
                           Cx<T> *__restrict__ out) {
    const size_t total = (size_t)Ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / Ngw), g = (int)(t - (size_t)b * Ngw);
        const Cx<T> p = psi[(size_t)b * ld + g], l = lam[(size_t)b * ld + g];
        out[t] = cadd(p, l);
        out[total + t] = cmake(p.x - l.x, p.y - l.y);
    }
}

template <typename T>
__global__ void k_zero(Cx<T> *p, int Ngw, int nb, int64_t ld) {
    const size_t total = (size_t)Ngw * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / Ngw), g = (int)(t - (size_t)b * Ngw);
        p[(size_t)b * ld + g] = cmake((T)0, (T)0);
    }
}


// ======================================================= fixed-size kernels
// The same passes with the line lengths as template constants (see
// pw_fft_tmpl.cuh); used for the grid sizes listed in FIXED_SIZES below,
// the run-time kernels above serve every other {2,3,5}-smooth size.
// FP32 lines use the register-fused composite radices (fewer shared-memory
// passes); FP64 lines here keep the 2/3/4/5/8 stages (register pressure in
// the z passes); the FP64 x-fused plane pass (kx_plane_vloc64) calls the
// fused plans directly with one CTA per SM.
template <typename T, int N, bool JF, bool PAD = false>
__device__ __forceinline__ void line_fft(Cx<T> *buf, int nl, int es, int ls, const Cx<T> *tw, int sign) {
    static_assert(!PAD || sizeof(T) == 4, "padded lines are FP32 only");
    if constexpr (sizeof(T) == 4)
        pwf::lines<T, N, JF, PAD>(buf, nl, es, ls, tw, sign);
    else
        pwt::lines<T, N, MaxV<T>::v, JF>(buf, nl, es, ls, tw, sign);
}

// natural index of shared twiddle entry i of an N-point line FFT of type T:
// the fused FP32 plans use their own layout (pwf::tw_src), the FP64 ones the
// natural table
template <typename T, int N> __device__ __forceinline__ int tw_src(int i) {
    if constexpr (sizeof(T) == 4)
        return pwf::tw_src<N>(i);
    else
        return i;
}

// Row stride (in elements) of the z-pass tile Z[kz][column] for Cg columns.
// The FP32 line FFTs run G = fp_group lines per warp with the line index
// fastest, so lane (line, j) reads word line + stride * j: a stride = G
// (mod 16) tiles the 16 eight-byte bank pairs for G < 16; with G >= 16
// (one line per lane) an odd stride keeps the entry scatter/gather, which
// walks kz down a column, off a single bank.  FP64 keeps Cg.
template <typename T, int N> __host__ __device__ constexpr int zrow(int Cg) {
    if constexpr (sizeof(T) == 8) {
        return Cg;
    } else {
        constexpr int G = pwf::fp_group<N>();
        return G >= 16 ? (Cg | 1) : Cg + ((G - Cg) % 16 + 16) % 16;
    }
}

template <typename T> struct MinBlocks;
template <> struct MinBlocks<float> { static constexpr int v = 2; };
template <> struct MinBlocks<double> { static constexpr int v = 2; };
// z passes: three CTAs per SM for every FP32 line length (80 registers, no
// spills; measured: Si216 FFT round trip 6.51 -> 6.31 ms against two CTAs)
template <typename T, int N3> struct ZBlocks { static constexpr int v = sizeof(T) == 4 ? 3 : 2; };

// z-pass bodies for one band: ps / hs its sphere coefficients, Ab its
// [z][column] block of the intermediate, column group blockIdx.x
constexpr int ZU = 4;   // sphere entries per thread per pass of the scatter / gather

// asynchronous global -> shared copies (no register staging, so a thread
// keeps every copy of a phase in flight at once)
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// z-passes of these line lengths stage through cp.async (measured: Si64
// round trip 0.657 -> 0.612 ms, Si216 8.50 -> 7.93 ms; the 27-point
// batched path was faster with register copies)
template <int N3> __host__ __device__ constexpr bool z_async() { return N3 >= 64; }

// one complex value: 8 bytes (FP32) or 16 bytes (FP64)
template <typename T> __device__ __forceinline__ void cp_async_cx(Cx<T> *smem, const Cx<T> *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
template <typename T, int N3>
__device__ __forceinline__ void zinv_band(const KPlan &kp, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ ps,
                                          Cx<T> *__restrict__ Ab, int Cg, int gx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *tw = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *Z = tw + N3;
    const int c0 = gx * Cg;
    const int cn = min(Cg, kp.Ncol - c0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int Zs = zrow<T, N3>(Cg);
    for (int i = threadIdx.x; i < N3; i += blockDim.x) tw[i] = twz[tw_src<T, N3>(i)];
    for (int i = threadIdx.x; i < N3 * Zs; i += blockDim.x) Z[i] = cmake((T)0, (T)0);
    __syncthreads();
    const int e0 = kp.col_ptr[c0], e1 = kp.col_ptr[c0 + cn];
    // ZU entries per thread per pass, every load issued before the first
    // use: the sphere reads are scattered and latency-bound
    for (int eb = e0 + threadIdx.x; eb < e1; eb += ZU * blockDim.x) {
        int ig[ZU], zi[ZU];
#pragma unroll
        for (int u = 0; u < ZU; ++u) {
            const int e = min(eb + u * (int)blockDim.x, e1 - 1);
            ig[u] = kp.ent_igw[e];
            zi[u] = kp.ent_kz[e] * Zs + kp.ent_col[e] - c0;
        }
        if constexpr (z_async<N3>()) {
#pragma unroll
            for (int u = 0; u < ZU; ++u)
                if (eb + u * (int)blockDim.x < e1) cp_async_cx<T>(&Z[zi[u]], &ps[ig[u]]);
        } else {
            Cx<T> pv[ZU];
#pragma unroll
            for (int u = 0; u < ZU; ++u) pv[u] = ps[ig[u]];
#pragma unroll
            for (int u = 0; u < ZU; ++u)
                if (eb + u * (int)blockDim.x < e1) Z[zi[u]] = pv[u];
        }
    }
    if constexpr (z_async<N3>()) cp_async_wait_all();
    __syncthreads();
    line_fft<T, N3, false>(Z, cn, Zs, 1, tw, +1);
    Ab += c0;
    for (int kz = warp; kz < N3; kz += nw)
        for (int cl = lane; cl < cn; cl += 32) Ab[(size_t)kz * kp.Ncol + cl] = Z[kz * Zs + cl];
}

template <typename T, int N3>
__global__ void __launch_bounds__(FFT_THREADS, ZBlocks<T, N3>::v)
kf_zinv(KPlan kp, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ psi, int64_t ld, Cx<T> *__restrict__ A,
        int Cg) {
    const int b = blockIdx.y;
    zinv_band<T, N3>(kp, twz, psi + (size_t)b * ld, A + (size_t)b * N3 * kp.Ncol, Cg, blockIdx.x);
}

template <typename T, int N3>
__device__ __forceinline__ void zfwd_band(const KPlan &kp, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ Ab,
                                          const Cx<T> *__restrict__ ps, Cx<T> *__restrict__ hs, int Cg, int flags, int gx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T> *tw = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *Z = tw + N3;
    const int c0 = gx * Cg;
    const int cn = min(Cg, kp.Ncol - c0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int Zs = zrow<T, N3>(Cg);
    for (int i = threadIdx.x; i < N3; i += blockDim.x) tw[i] = twz[tw_src<T, N3>(i)];
    Ab += c0;
    if constexpr (z_async<N3>()) {
        for (int kz = warp; kz < N3; kz += nw)
            for (int cl = lane; cl < cn; cl += 32) cp_async_cx<T>(&Z[kz * Zs + cl], &Ab[(size_t)kz * kp.Ncol + cl]);
        cp_async_wait_all();
    } else {
#pragma unroll 4
        for (int kz = warp; kz < N3; kz += nw)
            for (int cl = lane; cl < cn; cl += 32) Z[kz * Zs + cl] = Ab[(size_t)kz * kp.Ncol + cl];
    }
    __syncthreads();
    line_fft<T, N3, false>(Z, cn, Zs, 1, tw, -1);
    const int e0 = kp.col_ptr[c0], e1 = kp.col_ptr[c0 + cn];
    for (int eb = e0 + threadIdx.x; eb < e1; eb += ZU * blockDim.x) {
        int ig[ZU], zi[ZU];
#pragma unroll
        for (int u = 0; u < ZU; ++u) {
            const int e = min(eb + u * (int)blockDim.x, e1 - 1);
            ig[u] = kp.ent_igw[e];
            zi[u] = kp.ent_kz[e] * Zs + kp.ent_col[e] - c0;
        }
        Cx<T> kin[ZU], acc[ZU];
#pragma unroll
        for (int u = 0; u < ZU; ++u) {
            kin[u] = cmake((T)0, (T)0);
            acc[u] = cmake((T)0, (T)0);
            if (flags & 2) {
                const int e = min(eb + u * (int)blockDim.x, e1 - 1);
                const T g2 = sizeof(T) == 8 ? (T)kp.ent_g2[e] : (T)kp.ent_g2f[e];
                kin[u] = cscale(ps[ig[u]], (T)0.5 * g2);
            }
            if (flags & 4) acc[u] = hs[ig[u]];
        }
#pragma unroll
        for (int u = 0; u < ZU; ++u)
            if (eb + u * (int)blockDim.x < e1) {
                Cx<T> out = Z[zi[u]];
                if (flags & 2) out = cadd(out, kin[u]);
                if (flags & 4) out = cadd(out, acc[u]);
                hs[ig[u]] = out;
            }
    }
}

template <typename T, int N3>
__global__ void __launch_bounds__(FFT_THREADS, ZBlocks<T, N3>::v)
kf_zfwd(KPlan kp, const Cx<T> *__restrict__ twz, const Cx<T> *__restrict__ A, const Cx<T> *__restrict__ psi,
        Cx<T> *__restrict__ Hpsi, int64_t ld, int Cg, int flags) {
    const int b = blockIdx.y;
    zfwd_band<T, N3>(kp, twz, A + (size_t)b * N3 * kp.Ncol, psi + (size_t)b * ld, Hpsi + (size_t)b * ld, Cg, flags,
                     blockIdx.x);
}

template <typename T, int N1, int N2>
__device__ __forceinline__ void plane_to_real(const KPlan &kp, Cx<T> *S, Cx<T> *X, const Cx<T> *tx, int j0, int jc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = cmake((T)0, (T)0);
    __syncthreads();
    for (int ia = warp; ia < kp.Nxa; ia += nw) {
        const int x = kp.xa[ia];
        for (int jl = lane; jl < jc; jl += 32) X[jl * N1 + x] = S[ia * N2 + j0 + jl];
    }
    __syncthreads();
    line_fft<T, N1, true>(X, jc, 1, N1, tx, +1);
}

template <typename T, int N1, int N2>
__device__ __forceinline__ void plane_vloc_band(const KPlan &kp, const Cx<T> *__restrict__ twx,
                                                const Cx<T> *__restrict__ twy, const T *__restrict__ Vr,
                                                Cx<T> *__restrict__ Ab, int Jc, int kz) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Nxa = kp.Nxa, Ncol = kp.Ncol;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N1;
    Cx<T> *S = ty + N2;
    Cx<T> *X = S + Nxa * N2;
    
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[tw_src<T, N1>(i)];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[tw_src<T, N2>(i)];
    for (int i = threadIdx.x; i < Nxa * N2; i += blockDim.x) S[i] = cmake((T)0, (T)0);
    __syncthreads();
    Cx<T> *Ap = Ab + (size_t)kz * Ncol;
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
    __syncthreads();
    line_fft<T, N2, true>(S, Nxa, 1, N2, ty, +1);
    const T *Vp = Vr + (size_t)kz * N1 * N2;
    for (int j0 = 0; j0 < N2; j0 += Jc) {
        const int jc = min(Jc, N2 - j0);
        plane_to_real<T, N1, N2>(kp, S, X, tx, j0, jc);
        for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) X[i] = cscale(X[i], Vp[j0 * N1 + i]);
        __syncthreads();
        line_fft<T, N1, true>(X, jc, 1, N1, tx, -1);
        for (int ia = warp; ia < Nxa; ia += nw) {
            const int x = kp.xa[ia];
            for (int jl = lane; jl < jc; jl += 32) S[ia * N2 + j0 + jl] = X[jl * N1 + x];
        }
        __syncthreads();
    }
    line_fft<T, N2, true>(S, Nxa, 1, N2, ty, -1);
    for (int c = threadIdx.x; c < Ncol; c += blockDim.x) Ap[c] = S[kp.col_ia[c] * N2 + kp.col_j[c]];
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(FFT_THREADS, MinBlocks<T>::v)
kf_plane_vloc(KPlan kp, const Cx<T> *__restrict__ twx, const Cx<T> *__restrict__ twy, const T *__restrict__ Vr,
              Cx<T> *__restrict__ A, int Jc) {
    plane_vloc_band<T, N1, N2>(kp, twx, twy, Vr, A + (size_t)blockIdx.y * kp.N3 * kp.Ncol, Jc, blockIdx.x);
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(FFT_THREADS, MinBlocks<T>::v)
kf_plane_rho(KPlan kp, const Cx<T> *__restrict__ twx, const Cx<T> *__restrict__ twy, const Cx<T> *__restrict__ A,
             int nb, int Bg, const double *__restrict__ w, T *__restrict__ rho_part, int Jc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N3 = kp.N3, Nxa = kp.Nxa, Ncol = kp.Ncol;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N1;
    Cx<T> *S = ty + N2;
    Cx<T> *X = S + Nxa * N2;
    const int kz = blockIdx.x, g = blockIdx.y;
    constexpr int N12 = N1 * N2;
    T *rp = rho_part + (size_t)g * N12 * N3 + (size_t)kz * N12;
    for (int i = threadIdx.x; i < N1; i += blockDim.x) tx[i] = twx[tw_src<T, N1>(i)];
    for (int i = threadIdx.x; i < N2; i += blockDim.x) ty[i] = twy[tw_src<T, N2>(i)];
    for (int i = threadIdx.x; i < N12; i += blockDim.x) rp[i] = (T)0;
    const int b0 = g * Bg, b1 = min(nb, b0 + Bg);
    for (int b = b0; b < b1; ++b) {
        const T wb = (T)w[b];
        for (int i = threadIdx.x; i < Nxa * N2; i += blockDim.x) S[i] = cmake((T)0, (T)0);
        __syncthreads();
        const Cx<T> *Ap = A + ((size_t)b * N3 + kz) * Ncol;
        for (int c = threadIdx.x; c < Ncol; c += blockDim.x) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
        __syncthreads();
        line_fft<T, N2, true>(S, Nxa, 1, N2, ty, +1);
        for (int j0 = 0; j0 < N2; j0 += Jc) {
            const int jc = min(Jc, N2 - j0);
            plane_to_real<T, N1, N2>(kp, S, X, tx, j0, jc);
            for (int i = threadIdx.x; i < jc * N1; i += blockDim.x) {
                const Cx<T> v = X[i];
                rp[j0 * N1 + i] += wb * (v.x * v.x + v.y * v.y);
            }
            __syncthreads();
        }
    }
}


// ---------------------------------------------- FP32 plane kernels, x fused
// The x-direction work of a z-plane runs warp by warp on whole rows: the
// first stage of each inverse x-FFT reads the active-x entries of the
// sub-plane S directly (zeros elsewhere), the last stage multiplies by V(r)
// (op_V_loc) or accumulates w |psi(r)|^2 (calc_rhoe), and the last stage of
// the forward x-FFT writes only the active-x outputs back into S.  No block
// barrier is needed inside the x-pass, and the zero-fill, scatter, V and
// gather passes over the full plane disappear.

// shared-memory layout of the x-fused plane kernels (in float2 units)
struct PlaneXSmem {
    int N1, N2, Nxa, nwarps, group, plane_f;  // plane_f: floats of a full plane kept in shared memory (0 if none)
    int bands = 1;                            // sub-planes held at once (bands of the same z-plane)
    int xs = 0;                               // line stride of the per-warp x-line buffers (0: N1)
    int twn = -1;                             // twiddle entries (-1: N1 + N2)
    __host__ __device__ size_t elems() const {
        return (size_t)(twn >= 0 ? twn : N1 + N2) + (size_t)bands * Nxa * N2 + (size_t)nwarps * group * (xs ? xs : N1) +
               (plane_f + 1) / 2 + (N1 + 3) / 4;
    }
};

// Twiddle entries the x-fused op_V_loc kernel keeps: the fused plans read
// only exp(-2 pi i j / N), j < R0, at [R0, 2 R0) of the two-stage table
// (the radix DFTs hold their roots as constants, the other powers come from
// pwf::tw_pow); one-stage plans read none.  One table serves x and y.
template <int N> __host__ __device__ constexpr int xtw_lo() { return pwf::FPlan<N>::nst == 2 ? pwf::FPlan<N>::r(0) : 0; }
template <int N> __host__ __device__ constexpr int xtw_len() { return pwf::FPlan<N>::nst == 2 ? 2 * pwf::FPlan<N>::r(0) : 1; }

// Row y of the V(r) plane in shared memory starts at float vrow(y): rows 2m
// and 2m + 1 begin 15 words apart modulo 32, so the R0 = 15 consecutive x
// that the two half-warps of one x-pass read from two adjacent rows fall on
// 30 different banks (measured model of the 75-point kernel: 2 wavefronts
// per read with rows N1 apart, 1 with the gap).
template <int N1> __host__ __device__ constexpr int vgap() { return (15 - N1 % 32 + 32) % 32; }
template <int N1> __host__ __device__ constexpr int vrow(int y) { return y * N1 + vgap<N1>() * ((y + 1) >> 1); }
template <int N1, int N2> __host__ __device__ constexpr int vplane_floats() { return (vrow<N1>(N2) + 1) & ~1; }
// FP64 planes: the half-warps of an x-pass read 8-byte values, served one
// half-warp (one row) at a time, so no gap
template <typename T, int N1> __host__ __device__ constexpr int vrow_t(int y) {
    return sizeof(T) == 4 ? vrow<N1>(y) : y * N1;
}
template <typename T, int N1, int N2> __host__ __device__ constexpr int vplane_elems() {
    return sizeof(T) == 4 ? vplane_floats<N1, N2>() : N1 * N2;
}

// BPC sub-planes (nbh <= BPC bands of the same z-plane, band stride astr in
// A) go through every phase together: each block barrier then separates
// twice the line FFTs, and V(r), the twiddles and the active-x map are
// loaded once for all of them.
// Row stride of the sub-plane S: the line stride of the fused plan (elements
// of row ia at ia * LD + fp_pos(y)); the current plans are unpadded (on the
// 75-point grid padding would cost the third sub-plane per CTA).
template <int N> __host__ __device__ constexpr int plane_ld() { return pwf::fp_xs<N>(); }

template <typename T, int N1, int N2, bool VS, int BPC = 1>
__device__ __forceinline__ void plane_vloc_x_band(const KPlan &kp, const Cx<T> *__restrict__ twx,
                                                  const Cx<T> *__restrict__ twy, const T *__restrict__ Vr,
                                                  Cx<T> *__restrict__ Ab, int kz, int nbh = 1,
                                                  size_t astr = 0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    static_assert(N1 == N2, "one twiddle table serves x and y");
    (void)twy;
    constexpr int G = pwf::fp_group<N1>();
    const int Nxa = kp.Nxa, Ncol = kp.Ncol;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = FFT_THREADS / 32;
    Cx<T> *tw = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *S = tw + xtw_len<N1>();
    constexpr int LD = plane_ld<N2>();
    constexpr int XS = pwf::fp_xs<N1>();
    const size_t SP = (size_t)Nxa * LD;   // one sub-plane
    Cx<T> *Xw = S + BPC * SP + (size_t)warp * G * XS;
    T *Vs = reinterpret_cast<T *>(S + BPC * SP + (size_t)NW * G * XS);
    short *iax = reinterpret_cast<short *>(Vs + (VS ? vplane_elems<T, N1, N2>() : 0));

    const T *Vp = Vr + (size_t)kz * N1 * N2;
    if constexpr (VS) {
        for (int i = threadIdx.x; i < N1 * N2; i += FFT_THREADS) {
            T *dst = &Vs[vrow_t<T, N1>(i / N1) + i % N1];
            if constexpr (sizeof(T) == 4)
                cp_async4(dst, &Vp[i]);
            else
                cp_async_cx<float>(reinterpret_cast<Cx<float> *>(dst), reinterpret_cast<const Cx<float> *>(&Vp[i]));
        }
    }
    for (int i = threadIdx.x; i < N1; i += FFT_THREADS) iax[i] = -1;
    // the table of twx is in natural order: entry i of the fused layout is exp(-2 pi i tw_src(i) / N)
    for (int i = xtw_lo<N1>() + threadIdx.x; i < xtw_len<N1>(); i += FFT_THREADS) tw[i] = twx[pwf::tw_src<N1>(i)];
    for (int i = threadIdx.x; i < nbh * (int)SP; i += FFT_THREADS) S[i] = cmake((T)0, (T)0);
    __syncthreads();
    for (int i = threadIdx.x; i < Nxa; i += FFT_THREADS) iax[kp.xa[i]] = (short)i;
    for (int bb = 0; bb < nbh; ++bb) {
        const Cx<T> *Ap = Ab + bb * astr + (size_t)kz * Ncol;
        Cx<T> *Sb = S + bb * SP;
#pragma unroll 4
        for (int c = threadIdx.x; c < Ncol; c += FFT_THREADS) Sb[kp.col_ia[c] * LD + pwf::fp_pos<N2>(kp.col_j[c])] = Ap[c];
    }
    __syncthreads();
    // Two-stage plans: the R0 elements x = j + R1 r (r < R0) that this lane
    // reads in the first inverse x stage are the ones it writes in the last
    // forward stage (the same butterfly j = lane's slot in both), so their
    // active-x rows are looked up once, one byte each (255: x not active).
    constexpr bool TWO = pwf::FPlan<N1>::nst == 2;
    constexpr int XR0 = pwf::FPlan<N1>::r(0), XR1 = TWO ? pwf::FPlan<N1>::r(1) : 1;
    constexpr int NPK = TWO ? (XR0 + 3) / 4 : 1;
    unsigned pk[NPK];
    if constexpr (TWO) {
        static_assert(XR1 <= 16 && pwf::LaneMap<XR1, G>::ROUNDS == 1, "one x butterfly slot per lane");
        int ln, jl;
        pwf::LaneMap<XR1, G>::at(lane, 0, G, ln, jl);
#pragma unroll
        for (int w = 0; w < NPK; ++w) {
            unsigned u = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = 4 * w + b;
                const int ia = r < XR0 ? iax[jl + XR1 * r] : -1;
                u |= (unsigned)(ia >= 0 ? ia : 255) << (8 * b);
            }
            pk[w] = u;
        }
    }
    auto iax_at = [&](int x, int r) -> int {
        if constexpr (TWO) {
            (void)x;
            const int v = (pk[r >> 2] >> (8 * (r & 3))) & 255;
            return v == 255 ? -1 : v;
        } else {
            (void)r;
            return iax[x];
        }
    };
    pwf::lines<T, N2, true>(S, nbh * Nxa, 1, LD, tw, +1);  // ends with __syncthreads
    if constexpr (VS) {
        cp_async_wait_all();
        __syncthreads();
    }
    constexpr int NGRP = (N2 + G - 1) / G;
    for (int q = warp; q < nbh * NGRP; q += NW) {
        const int g0 = (q % NGRP) * G;
        Cx<T> *Sb = S + (q / NGRP) * SP;
        const int nl = min(G, N2 - g0);
        // rows g0 .. g0 + G - 1 lie in one padding block (G divides R0)
        static_assert(pwf::fp_pad<N2>() == 0 || pwf::FPlan<N2>::r(0) % G == 0, "row groups inside a padding block");
        const int yp = pwf::fp_pos<N2>(g0);
        auto ld_s = [&](int line, int x, int r) {
            const int ia = iax_at(x, r);
            return ia >= 0 ? Sb[ia * LD + yp + line] : cmake((T)0, (T)0);
        };
        auto vsc = [&](int line, int x) { return VS ? Vs[vrow_t<T, N1>(g0 + line) + x] : __ldg(&Vp[(g0 + line) * N1 + x]); };
        auto st_s = [&](int line, int x, int r, Cx<T> v) {
            const int ia = iax_at(x, r);
            if (ia >= 0) Sb[ia * LD + yp + line] = v;
        };
        pwf::group_fft_vpair<T, N1>(Xw, nl, tw, lane, ld_s, vsc, st_s);
    }
    __syncthreads();
    pwf::lines<T, N2, true>(S, nbh * Nxa, 1, LD, tw, -1);
    for (int bb = 0; bb < nbh; ++bb) {
        Cx<T> *Ap = Ab + bb * astr + (size_t)kz * Ncol;
        const Cx<T> *Sb = S + bb * SP;
#pragma unroll 4
        for (int c = threadIdx.x; c < Ncol; c += FFT_THREADS) Ap[c] = Sb[kp.col_ia[c] * LD + pwf::fp_pos<N2>(kp.col_j[c])];
    }
}

template <int N1, int N2, bool VS, int BPC>
__global__ void __launch_bounds__(FFT_THREADS, 2)
kx_plane_vloc(KPlan kp, const float2 *__restrict__ twx, const float2 *__restrict__ twy, const float *__restrict__ Vr,
              float2 *__restrict__ A, int nb) {
    const int b0 = blockIdx.y * BPC;
    const size_t astr = (size_t)kp.N3 * kp.Ncol;
    plane_vloc_x_band<float, N1, N2, VS, BPC>(kp, twx, twy, Vr, A + b0 * astr, blockIdx.x, min(BPC, nb - b0), astr);
}

// The same x-fused plane pass in FP64 (the reference's precision): the fused
// radix plans in double registers, one CTA per SM (up to 255 registers).
template <int N1, int N2, bool VS, int BPC>
__global__ void __launch_bounds__(FFT_THREADS, 1)
kx_plane_vloc64(KPlan kp, const double2 *__restrict__ twx, const double2 *__restrict__ twy,
                const double *__restrict__ Vr, double2 *__restrict__ A, int nb) {
    const int b0 = blockIdx.y * BPC;
    const size_t astr = (size_t)kp.N3 * kp.Ncol;
    plane_vloc_x_band<double, N1, N2, VS, BPC>(kp, twx, twy, Vr, A + b0 * astr, blockIdx.x, min(BPC, nb - b0), astr);
}

// calc_rhoe: bands [g*Bg, min(nb, (g+1)*Bg)) of plane kz; the weighted
// |psi(r)|^2 accumulate in shared memory when the plane fits (RS), else in
// the global partial sums directly.
template <typename T, int N1, int N2, bool RS>
__device__ __forceinline__ void plane_rho_x_body(const KPlan &kp, const Cx<T> *__restrict__ twx,
                                                 const Cx<T> *__restrict__ twy, const Cx<T> *__restrict__ A, int nb,
                                                 int Bg, const double *__restrict__ w, T *__restrict__ rho_part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int G = pwf::fp_group<N1>();
    constexpr int N12 = N1 * N2;
    const int N3 = kp.N3, Nxa = kp.Nxa, Ncol = kp.Ncol;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = FFT_THREADS / 32;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N1;
    Cx<T> *S = ty + N2;
    constexpr int XS = pwf::fp_xs<N1>();
    Cx<T> *Xw = S + Nxa * N2 + (size_t)warp * G * XS;
    T *Rs = reinterpret_cast<T *>(S + Nxa * N2 + (size_t)NW * G * XS);
    short *iax = reinterpret_cast<short *>(Rs + (RS ? N12 + (N12 & 1) : 0));
    const int kz = blockIdx.x, g = blockIdx.y;
    T *rp = rho_part + (size_t)g * N12 * N3 + (size_t)kz * N12;
    // the tables of twx, twy are in natural order (entry i of the fused layout: tw_src(i))
    for (int i = threadIdx.x; i < N1; i += FFT_THREADS) {
        tx[i] = twx[pwf::tw_src<N1>(i)];
        iax[i] = -1;
    }
    for (int i = threadIdx.x; i < N2; i += FFT_THREADS) ty[i] = twy[pwf::tw_src<N2>(i)];
    T *acc = RS ? Rs : rp;
    for (int i = threadIdx.x; i < N12; i += FFT_THREADS) acc[i] = (T)0;
    __syncthreads();
    for (int i = threadIdx.x; i < Nxa; i += FFT_THREADS) iax[kp.xa[i]] = (short)i;
    const int b0 = g * Bg, b1 = min(nb, b0 + Bg);
    for (int b = b0; b < b1; ++b) {
        const T wb = (T)w[b];
        for (int i = threadIdx.x; i < Nxa * N2; i += FFT_THREADS) S[i] = cmake((T)0, (T)0);
        __syncthreads();
        const Cx<T> *Ap = A + ((size_t)b * N3 + kz) * Ncol;
#pragma unroll 4
        for (int c = threadIdx.x; c < Ncol; c += FFT_THREADS) S[kp.col_ia[c] * N2 + kp.col_j[c]] = Ap[c];
        __syncthreads();
        pwf::lines<T, N2, true>(S, Nxa, 1, N2, ty, +1);
        for (int g0 = warp * G; g0 < N2; g0 += NW * G) {
            const int nl = min(G, N2 - g0);
            auto ld_s = [&](int line, int x, int) {
                const int ia = iax[x];
                return ia >= 0 ? S[ia * N2 + g0 + line] : cmake((T)0, (T)0);
            };
            auto st_r = [&](int line, int x, int, Cx<T> v) { acc[(g0 + line) * N1 + x] += wb * (v.x * v.x + v.y * v.y); };
            pwf::group_fft<T, N1>(Xw, nl, tx, +1, lane, ld_s, st_r);
        }
        __syncthreads();
    }
    if constexpr (RS)
        for (int i = threadIdx.x; i < N12; i += FFT_THREADS) rp[i] = Rs[i];
}

template <int N1, int N2, bool RS>
__global__ void __launch_bounds__(FFT_THREADS, 2)
kx_plane_rho(KPlan kp, const float2 *__restrict__ twx, const float2 *__restrict__ twy, const float2 *__restrict__ A,
             int nb, int Bg, const double *__restrict__ w, float *__restrict__ rho_part) {
    plane_rho_x_body<float, N1, N2, RS>(kp, twx, twy, A, nb, Bg, w, rho_part);
}

// The same x-fused density pass in FP64, one CTA per SM.
template <int N1, int N2, bool RS>
__global__ void __launch_bounds__(FFT_THREADS, 1)
kx_plane_rho64(KPlan kp, const double2 *__restrict__ twx, const double2 *__restrict__ twy, const double2 *__restrict__ A,
               int nb, int Bg, const double *__restrict__ w, double *__restrict__ rho_part) {
    plane_rho_x_body<double, N1, N2, RS>(kp, twx, twy, A, nb, Bg, w, rho_part);
}

// ------------------------------------------ batched op_H over k-points
// One launch per stage for the bands of many k-points (their Ngw, columns
// and active x differ): blockIdx.y is a band of the batch, band_k its
// k-point, whose plan, blocks and offset in A come from ks.  The band
// bodies are the single-k-point kernels' own.
template <typename T, int N3>
__global__ void __launch_bounds__(FFT_THREADS, ZBlocks<T, N3>::v)
mk_zinv(const MkK *__restrict__ ks, const int *__restrict__ band_k, const Cx<T> *__restrict__ twz, Cx<T> *__restrict__ A,
        int Cg) {
    const MkK &K = ks[band_k[blockIdx.y]];
    const KPlan kp = K.kp;
    if (blockIdx.x * Cg >= kp.Ncol) return;
    const int b = blockIdx.y - K.band0;
    zinv_band<T, N3>(kp, twz, (const Cx<T> *)K.psi + (size_t)b * K.ld, A + K.a_off + (size_t)b * N3 * kp.Ncol, Cg,
                     blockIdx.x);
}

template <typename T, int N3>
__global__ void __launch_bounds__(FFT_THREADS, ZBlocks<T, N3>::v)
mk_zfwd(const MkK *__restrict__ ks, const int *__restrict__ band_k, const Cx<T> *__restrict__ twz,
        const Cx<T> *__restrict__ A, int Cg, int flags) {
    const MkK &K = ks[band_k[blockIdx.y]];
    const KPlan kp = K.kp;
    if (blockIdx.x * Cg >= kp.Ncol) return;
    const int b = blockIdx.y - K.band0;
    zfwd_band<T, N3>(kp, twz, A + K.a_off + (size_t)b * N3 * kp.Ncol, (const Cx<T> *)K.psi + (size_t)b * K.ld,
                     (Cx<T> *)K.Hpsi + (size_t)b * K.ld, Cg, flags, blockIdx.x);
}

template <int N1, int N2, bool VS>
__global__ void __launch_bounds__(FFT_THREADS, 2)
mk_plane_vloc_x(const MkK *__restrict__ ks, const int *__restrict__ band_k, const float2 *__restrict__ twx,
                const float2 *__restrict__ twy, const float *__restrict__ Vr, float2 *__restrict__ A) {
    const MkK &K = ks[band_k[blockIdx.y]];
    const KPlan kp = K.kp;
    const int b = blockIdx.y - K.band0;
    plane_vloc_x_band<float, N1, N2, VS>(kp, twx, twy, Vr, A + K.a_off + (size_t)b * kp.N3 * kp.Ncol, blockIdx.x);
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(FFT_THREADS, MinBlocks<T>::v)
mk_plane_vloc(const MkK *__restrict__ ks, const int *__restrict__ band_k, const Cx<T> *__restrict__ twx,
              const Cx<T> *__restrict__ twy, const T *__restrict__ Vr, Cx<T> *__restrict__ A, int Jc) {
    const MkK &K = ks[band_k[blockIdx.y]];
    const KPlan kp = K.kp;
    const int b = blockIdx.y - K.band0;
    plane_vloc_band<T, N1, N2>(kp, twx, twy, Vr, A + K.a_off + (size_t)b * kp.N3 * kp.Ncol, Jc, blockIdx.x);
}

// Small cube grids whose lines fit one lane (single-stage register FFT, a
// warp holds all N lines of a direction): one warp per band, NW bands of
// the same z-plane per CTA sharing V(r) and the twiddles; every phase is
// warp-synchronous.  Lane l owns line l in each pass (y lines are the rows
// of the sub-plane S, x lines its columns), so no lane reads what another
// writes within a pass.
template <int N>
__device__ __forceinline__ void plane_vloc_w_body(const MkK *__restrict__ ks, const int *__restrict__ band_k, int nbands,
                                                  int nxa_max, const float2 *__restrict__ twx,
                                                  const float2 *__restrict__ twy, const float *__restrict__ Vr,
                                                  float2 *__restrict__ A, int kz, int bgroup) {
    static_assert(pwf::FPlan<N>::nst == 1 && pwf::fp_group<N>() >= N && pwf::fp_xs<N>() == N, "one line per lane");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using T = float;
    constexpr int NW = FFT_THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Cx<T> *tx = reinterpret_cast<Cx<T> *>(smem_raw);
    Cx<T> *ty = tx + N;
    float *Vs = reinterpret_cast<float *>(ty + N);
    Cx<T> *wbase = reinterpret_cast<Cx<T> *>(Vs + (N * N + 1) / 2 * 2);
    const size_t wsz = (size_t)nxa_max * N + (size_t)N * N + (N + 3) / 4;
    Cx<T> *S = wbase + (size_t)warp * wsz;
    Cx<T> *Xw = S + (size_t)nxa_max * N;
    short *iax = reinterpret_cast<short *>(Xw + N * N);
    for (int i = threadIdx.x; i < N * N; i += FFT_THREADS) Vs[i] = Vr[(size_t)kz * N * N + i];
    for (int i = threadIdx.x; i < N; i += FFT_THREADS) {
        tx[i] = twx[tw_src<float, N>(i)];
        ty[i] = twy[tw_src<float, N>(i)];
    }
    __syncthreads();
    const int gb = bgroup * NW + warp;
    if (gb >= nbands) return;
    const MkK &K = ks[band_k[gb]];
    const KPlan kp = K.kp;
    const int Nxa = kp.Nxa, Ncol = kp.Ncol;
    Cx<T> *Ap = A + K.a_off + ((size_t)(gb - K.band0) * N + kz) * Ncol;
    for (int x = lane; x < N; x += 32) iax[x] = -1;
    for (int i = lane; i < Nxa * N; i += 32) S[i] = cmake((T)0, (T)0);
    __syncwarp();
    for (int i = lane; i < Nxa; i += 32) iax[kp.xa[i]] = (short)i;
    for (int c = lane; c < Ncol; c += 32) S[kp.col_ia[c] * N + kp.col_j[c]] = Ap[c];
    __syncwarp();
    auto ld_row = [&](int line, int x, int) { return S[line * N + x]; };
    auto st_row = [&](int line, int x, int, Cx<T> v) { S[line * N + x] = v; };
    pwf::group_fft<T, N>(Xw, Nxa, ty, +1, lane, ld_row, st_row);
    __syncwarp();
    auto ld_s = [&](int line, int x, int) {
        const int ia = iax[x];
        return ia >= 0 ? S[ia * N + line] : cmake((T)0, (T)0);
    };
    auto vsc = [&](int line, int x) { return Vs[line * N + x]; };
    auto st_s = [&](int line, int x, int, Cx<T> v) {
        const int ia = iax[x];
        if (ia >= 0) S[ia * N + line] = v;
    };
    pwf::group_fft_vpair<T, N>(Xw, N, tx, lane, ld_s, vsc, st_s);
    __syncwarp();
    pwf::group_fft<T, N>(Xw, Nxa, ty, -1, lane, ld_row, st_row);
    __syncwarp();
    for (int c = lane; c < Ncol; c += 32) Ap[c] = S[kp.col_ia[c] * N + kp.col_j[c]];
}

template <int N>
__global__ void __launch_bounds__(FFT_THREADS)
mk_plane_vloc_w(const MkK *__restrict__ ks, const int *__restrict__ band_k, int nbands, int nxa_max,
                const float2 *__restrict__ twx, const float2 *__restrict__ twy, const float *__restrict__ Vr,
                float2 *__restrict__ A) {
    plane_vloc_w_body<N>(ks, band_k, nbands, nxa_max, twx, twy, Vr, A, blockIdx.x, blockIdx.y);
}

// op_V_Ps_nloc for small projector sets, one CTA per band of the batch:
// P = betaNL' psi (FP64 sums, one warp per projector), P2 = D P (the
// (ibeta, jbeta, h) list as CSR), Hpsi += betaNL P2
template <typename T>
__device__ __forceinline__ void vnl_body(const MkK *__restrict__ ks, const int *__restrict__ band_k,
                                         const int *__restrict__ Drow, const int *__restrict__ Dcol,
                                         const double *__restrict__ Dval, int nbeta, int band) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *P = reinterpret_cast<double2 *>(smem_raw);
    double2 *P2 = P + nbeta;
    const MkK &K = ks[band_k[band]];
    const int b = band - K.band0;
    const int ngw = K.kp.Ngw;
    const Cx<T> *beta = (const Cx<T> *)K.beta;
    const Cx<T> *ps = (const Cx<T> *)K.psi + (size_t)b * K.ld;
    Cx<T> *hs = (Cx<T> *)K.Hpsi + (size_t)b * K.ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = warp; j < nbeta; j += nw) {
        const Cx<T> *bj = beta + (size_t)j * ngw;
        // four independent partial sums per lane (latency, not bandwidth, bounds this loop)
        double r4[4] = {0.0, 0.0, 0.0, 0.0}, i4[4] = {0.0, 0.0, 0.0, 0.0};
        int g = lane;
        for (; g + 96 < ngw; g += 128) {
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const Cx<T> u = bj[g + 32 * t], v = ps[g + 32 * t];
                r4[t] += (double)u.x * v.x + (double)u.y * v.y;
                i4[t] += (double)u.x * v.y - (double)u.y * v.x;
            }
        }
        for (; g < ngw; g += 32) {
            const Cx<T> u = bj[g], v = ps[g];
            r4[0] += (double)u.x * v.x + (double)u.y * v.y;
            i4[0] += (double)u.x * v.y - (double)u.y * v.x;
        }
        double re = (r4[0] + r4[1]) + (r4[2] + r4[3]), im = (i4[0] + i4[1]) + (i4[2] + i4[3]);
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) P[j] = make_double2(re, im);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbeta; i += blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int e = Drow[i]; e < Drow[i + 1]; ++e) {
            re += Dval[e] * P[Dcol[e]].x;
            im += Dval[e] * P[Dcol[e]].y;
        }
        P2[i] = make_double2(re, im);
    }
    __syncthreads();
    for (int g = threadIdx.x; g < ngw; g += blockDim.x) {
        double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
        int i = 0;
        for (; i + 1 < nbeta; i += 2) {
            const Cx<T> u = beta[(size_t)i * ngw + g], w = beta[(size_t)(i + 1) * ngw + g];
            const double2 q = P2[i], r = P2[i + 1];
            re0 += (double)u.x * q.x - (double)u.y * q.y;
            im0 += (double)u.x * q.y + (double)u.y * q.x;
            re1 += (double)w.x * r.x - (double)w.y * r.y;
            im1 += (double)w.x * r.y + (double)w.y * r.x;
        }
        if (i < nbeta) {
            const Cx<T> u = beta[(size_t)i * ngw + g];
            const double2 q = P2[i];
            re0 += (double)u.x * q.x - (double)u.y * q.y;
            im0 += (double)u.x * q.y + (double)u.y * q.x;
        }
        const Cx<T> h = hs[g];
        hs[g] = cmake((T)(h.x + (re0 + re1)), (T)(h.y + (im0 + im1)));
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
mk_vnl(const MkK *__restrict__ ks, const int *__restrict__ band_k, const int *__restrict__ Drow,
       const int *__restrict__ Dcol, const double *__restrict__ Dval, int nbeta) {
    vnl_body<T>(ks, band_k, Drow, Dcol, Dval, nbeta, blockIdx.x);
}


// ------------------------------------ batched op_H in one persistent launch
// Every stage of the batched op_H (z inverse, plane pass, z forward, and the
// nonlocal part) in one cooperative launch: each phase is a grid-stride loop
// over its work items with the bodies of the per-stage kernels above, and a
// bounded grid barrier separates the phases (the plane pass needs every
// column of its z-plane, the forward z pass every plane of its columns, and
// the nonlocal part adds into the finished Hpsi).  The barrier counter is
// zeroed before the launch; a wait that gives up after PB_LIMIT polls records
// 3 in *err (read by pw_check_device) and the kernel runs to completion.
constexpr long long PB_LIMIT = 1ll << 22;
__device__ __forceinline__ void grid_bar(unsigned *ctr, unsigned &tgt, int *err) {
    __syncthreads();
    tgt += gridDim.x;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1u);
        if (!*(volatile int *)err) {
            long long it = 0;
            unsigned v;
            do {
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
                if (++it > PB_LIMIT) {
                    atomicExch(err, 3);
                    break;
                }
            } while (v < tgt);
        }
        __threadfence();
    }
    __syncthreads();
}

template <typename T, int NN>
__global__ void __launch_bounds__(FFT_THREADS, 2)
mk_persistent(const MkK *__restrict__ ks, const int *__restrict__ band_k, int nbands, int nxa_max, int max_ncol, int Cg,
              int Jc, const Cx<T> *__restrict__ twx, const Cx<T> *__restrict__ twy, const Cx<T> *__restrict__ twz,
              const T *__restrict__ Vr, Cx<T> *__restrict__ A, int flags, const int *__restrict__ Drow,
              const int *__restrict__ Dcol, const double *__restrict__ Dval, int nbeta, unsigned *ctr, int *err) {
    unsigned tgt = 0;
    const int ngx = (max_ncol + Cg - 1) / Cg;
    // z inverse: (column group, band)
#pragma unroll 1
    for (int q = blockIdx.x; q < ngx * nbands; q += gridDim.x) {
        const int gx = q % ngx, band = q / ngx;
        const MkK &K = ks[band_k[band]];
        const int b = band - K.band0;
        if (gx * Cg < K.kp.Ncol)
            zinv_band<T, NN>(K.kp, twz, (const Cx<T> *)K.psi + (size_t)b * K.ld, A + K.a_off + (size_t)b * NN * K.kp.Ncol,
                             Cg, gx);
        __syncthreads();
    }
    grid_bar(ctr, tgt, err);
    // plane pass: (z-plane, band) or, for one-lane lines, (z-plane, group of 8 bands)
    if constexpr (sizeof(T) == 4 && pwf::FPlan<NN>::nst == 1 && pwf::fp_group<NN>() >= NN) {
        constexpr int NW = FFT_THREADS / 32;
        const int ngroups = (nbands + NW - 1) / NW;
    #pragma unroll 1
    for (int q = blockIdx.x; q < NN * ngroups; q += gridDim.x) {
            plane_vloc_w_body<NN>(ks, band_k, nbands, nxa_max, twx, twy, Vr, A, q % NN, q / NN);
            __syncthreads();
        }
    } else {
    #pragma unroll 1
    for (int q = blockIdx.x; q < NN * nbands; q += gridDim.x) {
            const int kz = q % NN, band = q / NN;
            const MkK &K = ks[band_k[band]];
            Cx<T> *Ab = A + K.a_off + (size_t)(band - K.band0) * NN * K.kp.Ncol;
            if constexpr (sizeof(T) == 4) {
                constexpr bool VS = NN * NN * 4 <= 32 * 1024;
                plane_vloc_x_band<float, NN, NN, VS>(K.kp, twx, twy, Vr, Ab, kz);
            } else {
                plane_vloc_band<T, NN, NN>(K.kp, twx, twy, Vr, Ab, Jc, kz);
            }
            __syncthreads();
        }
    }
    grid_bar(ctr, tgt, err);
    // z forward with op_K and the gather into Hpsi
#pragma unroll 1
    for (int q = blockIdx.x; q < ngx * nbands; q += gridDim.x) {
        const int gx = q % ngx, band = q / ngx;
        const MkK &K = ks[band_k[band]];
        const int b = band - K.band0;
        if (gx * Cg < K.kp.Ncol)
            zfwd_band<T, NN>(K.kp, twz, A + K.a_off + (size_t)b * NN * K.kp.Ncol, (const Cx<T> *)K.psi + (size_t)b * K.ld,
                             (Cx<T> *)K.Hpsi + (size_t)b * K.ld, Cg, flags, gx);
        __syncthreads();
    }
    if (nbeta > 0) {
        grid_bar(ctr, tgt, err);
#pragma unroll 1
        for (int band = blockIdx.x; band < nbands; band += gridDim.x) {
            vnl_body<T>(ks, band_k, Drow, Dcol, Dval, nbeta, band);
            __syncthreads();
        }
    }
}
}  // namespace pwk

// ----------------------------------------------------------- host launchers
#include "pw_launch.h"

namespace pwk {

static int grid_stride_blocks(size_t total) {
    size_t b = (total + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

template <typename T>
static cudaError_t set_smem(const void *fn, size_t bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

// Line lengths with compile-time kernels (every dimension of the grids of
// the Si2/Al4 (27), Si64 (75) and Si216 (120) systems).
#define FIXED_SIZES(X) X(27) X(75) X(120)

template <typename T>
cudaError_t launch_zinv(const FftLaunch &L, const void *psi, int64_t ld, int nb, void *A, cudaStream_t st) {
    const KPlan &kp = L.kp;
    int Cg = L.Cg;
    size_t smem = (size_t)(kp.N3 + kp.N3 * Cg) * sizeof(Cx<T>);
    {
        dim3 grid((kp.Ncol + Cg - 1) / Cg, nb);
#define PW_CASE(NN)                                                                                                  \
    if (kp.N3 == NN) {                                                                                               \
        const size_t zsm = (size_t)(NN + NN * zrow<T, NN>(Cg)) * sizeof(Cx<T>);                                      \
        cudaError_t e = set_smem<T>((const void *)kf_zinv<T, NN>, zsm);                                              \
        if (e != cudaSuccess) return e;                                                                              \
        kf_zinv<T, NN><<<grid, FFT_THREADS, zsm, st>>>(kp, (const Cx<T> *)L.twz, (const Cx<T> *)psi, ld, (Cx<T> *)A, Cg); \
        return cudaGetLastError();                                                                                   \
    }
        FIXED_SIZES(PW_CASE)
#undef PW_CASE
    }
    cudaError_t e = set_smem<T>((const void *)k_zinv<T>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((kp.Ncol + Cg - 1) / Cg, nb);
    k_zinv<T><<<grid, FFT_THREADS, smem, st>>>(kp, L.dz, (const Cx<T> *)L.twz, (const Cx<T> *)psi, ld, (Cx<T> *)A, Cg);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_zfwd(const FftLaunch &L, const void *A, const void *psi, void *Hpsi, int64_t ld, int nb, int flags,
                        cudaStream_t st) {
    const KPlan &kp = L.kp;
    int Cg = L.Cg;
    size_t smem = (size_t)(kp.N3 + kp.N3 * Cg) * sizeof(Cx<T>);
    {
        dim3 grid((kp.Ncol + Cg - 1) / Cg, nb);
#define PW_CASE(NN)                                                                                                  \
    if (kp.N3 == NN) {                                                                                               \
        const size_t zsm = (size_t)(NN + NN * zrow<T, NN>(Cg)) * sizeof(Cx<T>);                                      \
        cudaError_t e = set_smem<T>((const void *)kf_zfwd<T, NN>, zsm);                                              \
        if (e != cudaSuccess) return e;                                                                              \
        kf_zfwd<T, NN><<<grid, FFT_THREADS, zsm, st>>>(kp, (const Cx<T> *)L.twz, (const Cx<T> *)A, (const Cx<T> *)psi, \
                                                        (Cx<T> *)Hpsi, ld, Cg, flags);                               \
        return cudaGetLastError();                                                                                   \
    }
        FIXED_SIZES(PW_CASE)
#undef PW_CASE
    }
    cudaError_t e = set_smem<T>((const void *)k_zfwd<T>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((kp.Ncol + Cg - 1) / Cg, nb);
    k_zfwd<T><<<grid, FFT_THREADS, smem, st>>>(kp, L.dz, (const Cx<T> *)L.twz, (const Cx<T> *)A, (const Cx<T> *)psi,
                                               (Cx<T> *)Hpsi, ld, Cg, flags);
    return cudaGetLastError();
}

// FP32 fixed sizes: the x-fused kernel (V(r) kept in shared memory when
// the plane takes at most 32 KB), BPC sub-planes per CTA
template <int NN, int BPC>
static cudaError_t launch_plane_vloc_xb(const FftLaunch &L, const void *Vr, void *A, int nb, cudaStream_t st) {
    const KPlan &kp = L.kp;
    constexpr bool VS = NN * NN * 4 <= 32 * 1024;
    PlaneXSmem ps{NN, plane_ld<NN>(), kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(), VS ? vplane_floats<NN, NN>() : 0};
    ps.bands = BPC;
    ps.xs = pwf::fp_xs<NN>();
    ps.twn = xtw_len<NN>();
    const size_t smem = ps.elems() * sizeof(float2);
    if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = set_smem<float>((const void *)kx_plane_vloc<NN, NN, VS, BPC>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, (nb + BPC - 1) / BPC);
    kx_plane_vloc<NN, NN, VS, BPC><<<grid, FFT_THREADS, smem, st>>>(kp, (const float2 *)L.twx, (const float2 *)L.twy,
                                                                   (const float *)Vr, (float2 *)A, nb);
    return cudaGetLastError();
}
// sub-planes per CTA (L.bpc), measured defaults: 3 on the 75-point grid
// (Si64 round trip 0.996 -> 0.843 ms); 1 on the 120-point grid (two CTAs per
// SM beat two sub-planes in one CTA: Si216 10.0 -> 8.7 ms with the earlier
// 24 * 5 plan); pw_autotune tries 1-3
template <int NN>
static cudaError_t launch_plane_vloc_x(const FftLaunch &L, const void *Vr, void *A, int nb, cudaStream_t st) {
    switch (L.bpc) {
        case 1: return launch_plane_vloc_xb<NN, 1>(L, Vr, A, nb, st);
        case 2: return launch_plane_vloc_xb<NN, 2>(L, Vr, A, nb, st);
        case 3: return launch_plane_vloc_xb<NN, 3>(L, Vr, A, nb, st);
        default: return cudaErrorInvalidValue;
    }
}
// FP64 x-fused plane pass on the two-stage grids (75, 120): V(r) in shared
// memory when the plane takes at most 48 KB, one band per CTA
template <int NN>
static cudaError_t launch_plane_vloc64_x(const FftLaunch &L, const void *Vr, void *A, int nb, cudaStream_t st) {
    const KPlan &kp = L.kp;
    constexpr bool VS = NN * NN * 8 <= 48 * 1024;
    PlaneXSmem ps{NN, plane_ld<NN>(), kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(), VS ? vplane_elems<double, NN, NN>() : 0};
    ps.bands = 1;
    ps.xs = pwf::fp_xs<NN>();
    ps.twn = xtw_len<NN>();
    const size_t smem = ps.elems() * sizeof(double2);
    if (smem > 227 * 1024) return cudaErrorNotSupported;   // the caller takes the plane-wide kernel
    cudaError_t e = set_smem<double>((const void *)kx_plane_vloc64<NN, NN, VS, 1>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, nb);
    kx_plane_vloc64<NN, NN, VS, 1><<<grid, FFT_THREADS, smem, st>>>(kp, (const double2 *)L.twx, (const double2 *)L.twy,
                                                                    (const double *)Vr, (double2 *)A, nb);
    return cudaGetLastError();
}
template <int NN>
static cudaError_t launch_plane_rho_x(const FftLaunch &L, const void *A, int nb, int G, int Bg, const double *w,
                                      void *rho_part, cudaStream_t st) {
    const KPlan &kp = L.kp;
    constexpr bool RS = NN * NN * 4 <= 32 * 1024;
    PlaneXSmem ps{NN, NN, kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(), RS ? NN * NN : 0};
    ps.xs = pwf::fp_xs<NN>();
    const size_t smem = ps.elems() * sizeof(float2);
    cudaError_t e = set_smem<float>((const void *)kx_plane_rho<NN, NN, RS>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, G);
    kx_plane_rho<NN, NN, RS><<<grid, FFT_THREADS, smem, st>>>(kp, (const float2 *)L.twx, (const float2 *)L.twy,
                                                             (const float2 *)A, nb, Bg, w, (float *)rho_part);
    return cudaGetLastError();
}

// FP64 x-fused density pass on the two-stage grids: the density plane in
// shared memory when it takes at most 48 KB, else the global partial sums
template <int NN>
static cudaError_t launch_plane_rho64_x(const FftLaunch &L, const void *A, int nb, int G, int Bg, const double *w,
                                        void *rho_part, cudaStream_t st) {
    const KPlan &kp = L.kp;
    constexpr bool RS = NN * NN * 8 <= 48 * 1024;
    PlaneXSmem ps{NN, NN, kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(), RS ? NN * NN : 0};
    ps.xs = pwf::fp_xs<NN>();
    const size_t smem = ps.elems() * sizeof(double2);
    if (smem > 227 * 1024) return cudaErrorNotSupported;   // the caller takes the plane-wide kernel
    cudaError_t e = set_smem<double>((const void *)kx_plane_rho64<NN, NN, RS>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, G);
    kx_plane_rho64<NN, NN, RS><<<grid, FFT_THREADS, smem, st>>>(kp, (const double2 *)L.twx, (const double2 *)L.twy,
                                                               (const double2 *)A, nb, Bg, w, (double *)rho_part);
    return cudaGetLastError();
}

// Batched op_H stages over the bands of many k-points (cube grids of the
// compiled sizes).  L: twiddles, Cg and Jc of the k-point with the most
// active x (sizes the plane pass's shared memory); max_ncol sizes the z
// grids.  flags as kf_zfwd (2: + op_K, 4: accumulate).
template <typename T>
cudaError_t launch_multik(const FftLaunch &L, const MkK *ks, const int *band_k, int nk, int nbands, int max_nb,
                          int max_ncol, const void *Vr, void *A, int flags, const int *Drow, const int *Dcol,
                          const double *Dval, int nbeta, cudaStream_t st) {
    const KPlan &kp = L.kp;
    if (kp.N1 != kp.N2 || kp.N2 != kp.N3) return cudaErrorNotSupported;
    const int Cg = L.Cg;
    const dim3 zgrid((max_ncol + Cg - 1) / Cg, nbands);
    cudaError_t e = cudaErrorNotSupported;
#define PW_CASE(NN)                                                                                                  \
    if (kp.N1 == NN) {                                                                                               \
        const size_t zsm = (size_t)(NN + NN * zrow<T, NN>(Cg)) * sizeof(Cx<T>);                                      \
        if ((e = set_smem<T>((const void *)mk_zinv<T, NN>, zsm)) != cudaSuccess) return e;                          \
        mk_zinv<T, NN><<<zgrid, FFT_THREADS, zsm, st>>>(ks, band_k, (const Cx<T> *)L.twz, (Cx<T> *)A, Cg);           \
        if ((e = cudaGetLastError()) != cudaSuccess) return e;                                                       \
        if constexpr (sizeof(T) == 4 && pwf::FPlan<NN>::nst == 1 && pwf::fp_group<NN>() >= NN) {                    \
            const size_t psm = (2 * NN + (NN * NN + 1) / 2) * sizeof(float2) +                                       \
                               (FFT_THREADS / 32) * ((size_t)kp.Nxa * NN + NN * NN + (NN + 3) / 4) * sizeof(float2); \
            if ((e = set_smem<float>((const void *)mk_plane_vloc_w<NN>, psm)) != cudaSuccess) return e;             \
            mk_plane_vloc_w<NN><<<dim3(NN, (nbands + FFT_THREADS / 32 - 1) / (FFT_THREADS / 32)), FFT_THREADS, psm,  \
                                  st>>>(ks, band_k, nbands, kp.Nxa, (const float2 *)L.twx, (const float2 *)L.twy,   \
                                        (const float *)Vr, (float2 *)A);                                             \
        } else if constexpr (sizeof(T) == 4) {                                                                       \
            constexpr bool VS = NN * NN * 4 <= 32 * 1024;                                                            \
            PlaneXSmem ps{NN, plane_ld<NN>(), kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(),                         \
                          VS ? vplane_floats<NN, NN>() : 0};                                                         \
            ps.xs = pwf::fp_xs<NN>();                                                                                \
            ps.twn = xtw_len<NN>();                                                                                  \
            const size_t psm = ps.elems() * sizeof(float2);                                                          \
            if ((e = set_smem<float>((const void *)mk_plane_vloc_x<NN, NN, VS>, psm)) != cudaSuccess) return e;     \
            mk_plane_vloc_x<NN, NN, VS><<<dim3(NN, nbands), FFT_THREADS, psm, st>>>(                                 \
                ks, band_k, (const float2 *)L.twx, (const float2 *)L.twy, (const float *)Vr, (float2 *)A);          \
        } else {                                                                                                     \
            const PlaneSmem ps{NN, NN, kp.Nxa, L.Jc};                                                                \
            const size_t psm = ps.elems() * sizeof(Cx<T>);                                                           \
            if ((e = set_smem<T>((const void *)mk_plane_vloc<T, NN, NN>, psm)) != cudaSuccess) return e;            \
            mk_plane_vloc<T, NN, NN><<<dim3(NN, nbands), FFT_THREADS, psm, st>>>(                                    \
                ks, band_k, (const Cx<T> *)L.twx, (const Cx<T> *)L.twy, (const T *)Vr, (Cx<T> *)A, L.Jc);           \
        }                                                                                                            \
        if ((e = cudaGetLastError()) != cudaSuccess) return e;                                                       \
        if ((e = set_smem<T>((const void *)mk_zfwd<T, NN>, zsm)) != cudaSuccess) return e;                          \
        mk_zfwd<T, NN><<<zgrid, FFT_THREADS, zsm, st>>>(ks, band_k, (const Cx<T> *)L.twz, (const Cx<T> *)A, Cg,      \
                                                        flags);                                                      \
        if ((e = cudaGetLastError()) != cudaSuccess) return e;                                                       \
    }
    FIXED_SIZES(PW_CASE)
#undef PW_CASE
    if (e != cudaSuccess) return e;
    if (nbeta > 0) {
        const size_t vsm = 2 * (size_t)nbeta * sizeof(double2);
        if ((e = set_smem<T>((const void *)mk_vnl<T>, vsm)) != cudaSuccess) return e;
        mk_vnl<T><<<nbands, 256, vsm, st>>>(ks, band_k, Drow, Dcol, Dval, nbeta);
        e = cudaGetLastError();
    }
    return e;
}


// The batched op_H of launch_multik as one cooperative launch of
// mk_persistent (as many CTAs as fit on the GPU at once, each looping over
// work items).  ctr: a device counter (zeroed here), err: the context's
// error word.  cudaErrorCooperativeLaunchTooLarge when one CTA per SM does
// not fit (the caller then runs launch_multik).
template <typename T>
cudaError_t launch_multik_persistent(const FftLaunch &L, const MkK *ks, const int *band_k, int nbands, int max_ncol,
                                     const void *Vr, void *A, int flags, const int *Drow, const int *Dcol,
                                     const double *Dval, int nbeta, unsigned *ctr, int *err, cudaStream_t st) {
    const KPlan &kp = L.kp;
    if (kp.N1 != kp.N2 || kp.N2 != kp.N3) return cudaErrorNotSupported;
    const int Cg = L.Cg;
    cudaError_t e = cudaErrorNotSupported;
#define PW_CASE(NN)                                                                                                  \
    if (kp.N1 == NN) {                                                                                               \
        size_t sm = (size_t)(NN + NN * zrow<T, NN>(Cg)) * sizeof(Cx<T>);                                             \
        if constexpr (sizeof(T) == 4 && pwf::FPlan<NN>::nst == 1 && pwf::fp_group<NN>() >= NN) {                    \
            sm = std::max(sm, (2 * NN + (NN * NN + 1) / 2) * sizeof(float2) +                                         \
                                  (FFT_THREADS / 32) * ((size_t)kp.Nxa * NN + NN * NN + (NN + 3) / 4) * sizeof(float2)); \
        } else if constexpr (sizeof(T) == 4) {                                                                       \
            constexpr bool VS = NN * NN * 4 <= 32 * 1024;                                                            \
            PlaneXSmem ps{NN, plane_ld<NN>(), kp.Nxa, FFT_THREADS / 32, pwf::fp_group<NN>(),                         \
                          VS ? vplane_floats<NN, NN>() : 0};                                                         \
            ps.xs = pwf::fp_xs<NN>();                                                                                \
            ps.twn = xtw_len<NN>();                                                                                  \
            sm = std::max(sm, ps.elems() * sizeof(float2));                                                          \
        } else {                                                                                                     \
            const PlaneSmem ps{NN, NN, kp.Nxa, L.Jc};                                                                \
            sm = std::max(sm, ps.elems() * sizeof(Cx<T>));                                                           \
        }                                                                                                            \
        sm = std::max(sm, 2 * (size_t)nbeta * sizeof(double2));                                                      \
        const void *fn = (const void *)mk_persistent<T, NN>;                                                         \
        if ((e = set_smem<T>(fn, sm)) != cudaSuccess) return e;                                                      \
        int dev = 0, sms = 0, per = 0;                                                                               \
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;                                                      \
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;        \
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, FFT_THREADS, sm)) != cudaSuccess) return e; \
        if (per < 1) return cudaErrorCooperativeLaunchTooLarge;                                                      \
        if ((e = cudaMemsetAsync(ctr, 0, sizeof(unsigned), st)) != cudaSuccess) return e;                            \
        const int ngx = (max_ncol + Cg - 1) / Cg;                                                                    \
        const int nblk = std::max(1, std::min(sms * per, ngx * nbands));                                            \
        const int nxa = kp.Nxa, Jc = L.Jc;                                                                           \
        const Cx<T> *tx = (const Cx<T> *)L.twx, *ty = (const Cx<T> *)L.twy, *tz = (const Cx<T> *)L.twz;             \
        const T *V = (const T *)Vr;                                                                                  \
        Cx<T> *Ap = (Cx<T> *)A;                                                                                      \
        void *args[] = {(void *)&ks, (void *)&band_k, (void *)&nbands, (void *)&nxa, (void *)&max_ncol, (void *)&Cg, \
                        (void *)&Jc, (void *)&tx, (void *)&ty, (void *)&tz, (void *)&V, (void *)&Ap, (void *)&flags, \
                        (void *)&Drow, (void *)&Dcol, (void *)&Dval, (void *)&nbeta, (void *)&ctr, (void *)&err};    \
        return cudaLaunchCooperativeKernel(fn, nblk, FFT_THREADS, args, sm, st);                                     \
    }
    FIXED_SIZES(PW_CASE)
#undef PW_CASE
    return e;
}

template <typename T>
cudaError_t launch_plane_vloc(const FftLaunch &L, const void *Vr, void *A, int nb, cudaStream_t st) {
    const KPlan &kp = L.kp;
    if constexpr (sizeof(T) == 4) {
        if (kp.N1 == kp.N2) {
#define PW_CASE(NN) \
    if (kp.N1 == NN) return launch_plane_vloc_x<NN>(L, Vr, A, nb, st);
            FIXED_SIZES(PW_CASE)
#undef PW_CASE
        }
    } else if (kp.N1 == kp.N2 && (kp.N1 == 75 || kp.N1 == 120)) {
        // x-fused when its sub-plane fits in shared memory (active x up to ~80 of 120)
        const cudaError_t e = kp.N1 == 75 ? launch_plane_vloc64_x<75>(L, Vr, A, nb, st)
                                          : launch_plane_vloc64_x<120>(L, Vr, A, nb, st);
        if (e != cudaErrorNotSupported) return e;
    }
    PlaneSmem ps{kp.N1, kp.N2, kp.Nxa, L.Jc};
    size_t smem = ps.elems() * sizeof(Cx<T>);
    if (kp.N1 == kp.N2) {
        dim3 grid(kp.N3, nb);
#define PW_CASE(NN)                                                                                                  \
    if (kp.N1 == NN) {                                                                                               \
        cudaError_t e = set_smem<T>((const void *)kf_plane_vloc<T, NN, NN>, smem);                                   \
        if (e != cudaSuccess) return e;                                                                              \
        kf_plane_vloc<T, NN, NN><<<grid, FFT_THREADS, smem, st>>>(kp, (const Cx<T> *)L.twx, (const Cx<T> *)L.twy,    \
                                                                  (const T *)Vr, (Cx<T> *)A, L.Jc);                  \
        return cudaGetLastError();                                                                                   \
    }
        FIXED_SIZES(PW_CASE)
#undef PW_CASE
    }
    cudaError_t e = set_smem<T>((const void *)k_plane_vloc<T>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, nb);
    k_plane_vloc<T><<<grid, FFT_THREADS, smem, st>>>(kp, L.dx, L.dy, (const Cx<T> *)L.twx, (const Cx<T> *)L.twy,
                                                     (const T *)Vr, (Cx<T> *)A, L.Jc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_plane_rho(const FftLaunch &L, const void *A, int nb, int G, int Bg, const double *w, void *rho_part,
                             cudaStream_t st) {
    const KPlan &kp = L.kp;
    if constexpr (sizeof(T) == 4) {
        if (kp.N1 == kp.N2) {
#define PW_CASE(NN) \
    if (kp.N1 == NN) return launch_plane_rho_x<NN>(L, A, nb, G, Bg, w, rho_part, st);
            FIXED_SIZES(PW_CASE)
#undef PW_CASE
        }
    } else if (kp.N1 == kp.N2 && (kp.N1 == 75 || kp.N1 == 120)) {
        const cudaError_t e = kp.N1 == 75 ? launch_plane_rho64_x<75>(L, A, nb, G, Bg, w, rho_part, st)
                                          : launch_plane_rho64_x<120>(L, A, nb, G, Bg, w, rho_part, st);
        if (e != cudaErrorNotSupported) return e;
    }
    PlaneSmem ps{kp.N1, kp.N2, kp.Nxa, L.Jc};
    size_t smem = ps.elems() * sizeof(Cx<T>);
    if (kp.N1 == kp.N2) {
        dim3 grid(kp.N3, G);
#define PW_CASE(NN)                                                                                                  \
    if (kp.N1 == NN) {                                                                                               \
        cudaError_t e = set_smem<T>((const void *)kf_plane_rho<T, NN, NN>, smem);                                    \
        if (e != cudaSuccess) return e;                                                                              \
        kf_plane_rho<T, NN, NN><<<grid, FFT_THREADS, smem, st>>>(kp, (const Cx<T> *)L.twx, (const Cx<T> *)L.twy,     \
                                                                 (const Cx<T> *)A, nb, Bg, w, (T *)rho_part, L.Jc);  \
        return cudaGetLastError();                                                                                   \
    }
        FIXED_SIZES(PW_CASE)
#undef PW_CASE
    }
    cudaError_t e = set_smem<T>((const void *)k_plane_rho<T>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(kp.N3, G);
    k_plane_rho<T><<<grid, FFT_THREADS, smem, st>>>(kp, L.dx, L.dy, (const Cx<T> *)L.twx, (const Cx<T> *)L.twy,
                                                    (const Cx<T> *)A, nb, Bg, w, (T *)rho_part, L.Jc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_rho_reduce(const void *part, int G, size_t N, double *rho, int accumulate, cudaStream_t st) {
    k_rho_reduce<T><<<grid_stride_blocks(N), 256, 0, st>>>((const T *)part, G, N, rho, accumulate);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_opK(int Ngw, int nb, const double *Gk2, const void *psi, void *Hpsi, int64_t ld, int accumulate,
                       cudaStream_t st) {
    k_opK<T><<<grid_stride_blocks((size_t)Ngw * nb), 256, 0, st>>>(Ngw, nb, Gk2, (const Cx<T> *)psi, (Cx<T> *)Hpsi, ld,
                                                                   accumulate);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_kprec(int Ngw, int nb, const double *Gk2, const void *in, void *out, int64_t ld, cudaStream_t st) {
    k_kprec<T><<<grid_stride_blocks((size_t)Ngw * nb), 256, 0, st>>>(Ngw, nb, Gk2, (const Cx<T> *)in, (Cx<T> *)out, ld);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_polarize(int Ngw, int nb, const void *psi, const void *lam, int64_t ld, void *out, cudaStream_t st) {
    k_polarize<T><<<grid_stride_blocks((size_t)Ngw * nb), 256, 0, st>>>(Ngw, nb, (const Cx<T> *)psi, (const Cx<T> *)lam,
                                                                         ld, (Cx<T> *)out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_zero(void *p, int Ngw, int nb, int64_t ld, cudaStream_t st) {
    k_zero<T><<<grid_stride_blocks((size_t)Ngw * nb), 256, 0, st>>>((Cx<T> *)p, Ngw, nb, ld);
    return cudaGetLastError();
}

#define PW_INST(T)                                                                                                   \
    template cudaError_t launch_zinv<T>(const FftLaunch &, const void *, int64_t, int, void *, cudaStream_t);       \
    template cudaError_t launch_zfwd<T>(const FftLaunch &, const void *, const void *, void *, int64_t, int, int,  \
                                        cudaStream_t);                                                               \
    template cudaError_t launch_plane_vloc<T>(const FftLaunch &, const void *, void *, int, cudaStream_t);          \
    template cudaError_t launch_multik_persistent<T>(const FftLaunch &, const MkK *, const int *, int, int,          \
                                                     const void *, void *, int, const int *, const int *,          \
                                                     const double *, int, unsigned *, int *, cudaStream_t);         \
    template cudaError_t launch_multik<T>(const FftLaunch &, const MkK *, const int *, int, int, int, int,           \
                                          const void *, void *, int, const int *, const int *, const double *, int,  \
                                          cudaStream_t);                                                             \
    template cudaError_t launch_plane_rho<T>(const FftLaunch &, const void *, int, int, int, const double *, void *, \
                                             cudaStream_t);                                                          \
    template cudaError_t launch_rho_reduce<T>(const void *, int, size_t, double *, int, cudaStream_t);              \
    template cudaError_t launch_opK<T>(int, int, const double *, const void *, void *, int64_t, int, cudaStream_t); \
    template cudaError_t launch_kprec<T>(int, int, const double *, const void *, void *, int64_t, cudaStream_t);    \
    template cudaError_t launch_zero<T>(void *, int, int, int64_t, cudaStream_t);                                \
    template cudaError_t launch_polarize<T>(int, int, const void *, const void *, int64_t, void *, cudaStream_t);
PW_INST(float)
PW_INST(double)

}  // namespace pwk
