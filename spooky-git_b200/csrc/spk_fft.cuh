// spk_fft.cuh -- complex helpers and in-register DFT butterflies for the
// SPOOKY FFT passes (sm_100a).
//
// dft2/4/8/16 compute, in registers and in natural order,
//     X[t] = sum_r x[r] exp(DIR * 2*pi*i * r*t / R)      (DIR = -1 forward),
// written from the DFT definition as nested radix-2 splittings; the
// register-resident transforms of spk_regfft.cuh are built from them.
// FftPlan carries the length of an axis and its twiddle table W_N^k
// (computed on the host in extended precision).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace spk {

template <typename T> struct cx;
template <> struct cx<float>  { using t = float2; };
template <> struct cx<double> { using t = double2; };
template <typename T> using C2 = typename cx<T>::t;

template <typename T> __device__ __forceinline__ C2<T> mk(T x, T y) { C2<T> r; r.x = x; r.y = y; return r; }
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename V> __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename S> __device__ __forceinline__ V cscale(S s, V a) { a.x *= s; a.y *= s; return a; }
// multiply by DIR*i  (DIR=-1: -i, DIR=+1: +i)
template <int DIR, typename V> __device__ __forceinline__ V rot90(V a) {
    V r;
    if (DIR < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
    return r;
}
// a * (c + DIR*i*s)
template <int DIR, typename V, typename T> __device__ __forceinline__ V rotc(V a, T c, T s) {
    V r;
    if (DIR < 0) { r.x = a.x * c + a.y * s; r.y = a.y * c - a.x * s; }
    else         { r.x = a.x * c - a.y * s; r.y = a.y * c + a.x * s; }
    return r;
}

// FP32 complex arithmetic on Blackwell's paired FP32 instructions (FADD2,
// FMUL2, FFMA2: one instruction for both lanes, each lane rounded as the
// scalar operation).  Sums, differences and real scalings give the same bits
// as the scalar forms; the products round a.x b (both lanes) first and fuse
// the a.y terms, the same single-FMA accuracy as the scalar contraction.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as fma(-1, b, a): exact product, one rounding -- the bits of a - b
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }
__device__ __forceinline__ float2 cscale(float s, float2 a) { return __fmul2_rn(make_float2(s, s), a); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    // (a.x b.x - a.y b.y, a.x b.y + a.y b.x)
    return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}
template <int DIR> __device__ __forceinline__ float2 rotc(float2 a, float c, float s) {
    // DIR < 0: (a.x c + a.y s, a.y c - a.x s); DIR > 0: (a.x c - a.y s, a.y c + a.x s)
    const float2 t = __fmul2_rn(a, make_float2(c, c));
    return DIR < 0 ? __ffma2_rn(make_float2(a.y, -a.x), make_float2(s, s), t)
                   : __ffma2_rn(make_float2(-a.y, a.x), make_float2(s, s), t);
}
#endif

// ---- in-register DFTs (natural-order input and output) -------------------
template <typename T, int DIR> __device__ __forceinline__ void dft2(C2<T>* a) {
    C2<T> t = a[0]; a[0] = cadd(t, a[1]); a[1] = csub(t, a[1]);
}
template <typename T, int DIR> __device__ __forceinline__ void dft4(C2<T>* a) {
    C2<T> s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
    C2<T> s13 = cadd(a[1], a[3]), d13 = rot90<DIR>(csub(a[1], a[3]));
    a[0] = cadd(s02, s13); a[2] = csub(s02, s13);
    a[1] = cadd(d02, d13); a[3] = csub(d02, d13);
}
template <typename T, int DIR> __device__ __forceinline__ void dft8(C2<T>* a) {
    const T h = (T)0.70710678118654752440;   // cos(pi/4)
    C2<T> e[4] = {a[0], a[2], a[4], a[6]};
    C2<T> o[4] = {a[1], a[3], a[5], a[7]};
    dft4<T, DIR>(e); dft4<T, DIR>(o);
    o[1] = rotc<DIR>(o[1], h, h);
    o[2] = rot90<DIR>(o[2]);
    o[3] = rotc<DIR>(o[3], -h, h);
#pragma unroll
    for (int k = 0; k < 4; k++) { a[k] = cadd(e[k], o[k]); a[k + 4] = csub(e[k], o[k]); }
}
template <typename T, int DIR> __device__ __forceinline__ void dft16(C2<T>* a) {
    const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;   // cos, sin(pi/8)
    const T h = (T)0.70710678118654752440;
    C2<T> e[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; k++) { e[k] = a[2 * k]; o[k] = a[2 * k + 1]; }
    dft8<T, DIR>(e); dft8<T, DIR>(o);
    o[1] = rotc<DIR>(o[1], c1, s1);
    o[2] = rotc<DIR>(o[2], h, h);
    o[3] = rotc<DIR>(o[3], s1, c1);
    o[4] = rot90<DIR>(o[4]);
    o[5] = rotc<DIR>(o[5], -s1, c1);
    o[6] = rotc<DIR>(o[6], -h, h);
    o[7] = rotc<DIR>(o[7], -c1, s1);
#pragma unroll
    for (int k = 0; k < 8; k++) { a[k] = cadd(e[k], o[k]); a[k + 8] = csub(e[k], o[k]); }
}

// One axis length and its twiddle table W_N^k.
struct FftPlan {
    int n;
    const void* tw;   // C2<T>[n]: exp(-2 pi i k/n), in the pass precision
};

// Element n of a column at n (PAD = 0) or n + n/16 (PAD = 1: one pad slot
// per 16 elements breaks the stride-R bank conflicts of contiguous columns).
template <int PAD> __device__ __forceinline__ int padi(int n) { return PAD ? n + (n >> 4) : n; }
// n plus one pad element per block of B (a power of two), n >= 0
template <int B> __device__ __forceinline__ int padb(int n) { return n + (int)((unsigned)n / (unsigned)B); }
__host__ __device__ inline int padded_len(int n) { return n + (n >> 4); }

__host__ __device__ inline int ilog2(int n) { int l = 0; while ((1 << l) < n) l++; return l; }


}  // namespace spk
