// Shared device helpers: complex arithmetic on float2/double2 and the
// per-k-point pruned-FFT tables handed to the kernels by value.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using Cx = typename CplxOf<T>::type;

__host__ __device__ __forceinline__ float2 cmake(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 cmake(double a, double b) { return make_double2(a, b); }

template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { return cmake(a.x + b.x, a.y + b.y); }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { return cmake(a.x - b.x, a.y - b.y); }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    return cmake(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    return cmake(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) { return cmake(a.x * s, a.y * s); }
// i * s * a  (s = +1 or -1)
template <typename V, typename S> __host__ __device__ __forceinline__ V cmul_is(V a, S s) { return cmake(-a.y * s, a.x * s); }

// One FFT dimension: length and its radix plan (radices 2,3,4,5,8).
struct FftDim {
    int n;
    int nstage;
    int radix[12];
};

// Grid-wide constants for the pruned transforms of one k-point.
struct KPlan {
    int N1, N2, N3;
    int Ngw;            // sphere points
    int Ncol;           // active (x,y) columns
    int Nxa;            // active x indices
    const int *col_ptr;    // [Ncol+1] CSR into the ent_* arrays (column-sorted)
    const int *ent_igw;    // [Ngw] sphere index of entry
    const int *ent_kz;     // [Ngw] z index of entry
    const int *ent_col;    // [Ngw] column of entry
    const int *col_ia;     // [Ncol] position of the column's x in the active-x list
    const int *col_j;      // [Ncol] y index of the column
    const int *xa;         // [Nxa] active x values
    const double *Gk2;     // [Ngw] |G+k|^2
    const float *Gk2f;     // [Ngw] |G+k|^2 (FP32 copy)
    const double *ent_g2;  // [Ngw] |G+k|^2 of entry e (entry order: coalesced in the z passes)
    const float *ent_g2f;  // [Ngw] FP32 copy
};

// One k-point of a batched op_H (every k-point and band in one launch per
// stage): its plan, its blocks, where its bands start in the batch's band
// list and in the intermediate A, and its projectors.
struct MkK {
    KPlan kp;
    const void *psi;    // Ngw x nb (ld), launch precision
    void *Hpsi;         // Ngw x nb (ld)
    const void *beta;   // Ngw x nbeta projectors (ld Ngw), launch precision; null: no V_NL
    int64_t ld;
    size_t a_off;       // element offset of the k-point's band 0 in A
    int band0, nb;
};
