// spk_fft.cuh -- shared-memory mixed-radix FFT for the SPOOKY passes (sm_100a).
//
// A CTA transforms `ncol` independent sequences of length N held in shared
// memory; element (n, col) lives at buf[n*es + col*cs].  The transform is a
// Stockham decimation-in-frequency FFT written from the DFT definition
//     X[t] = sum_n x[n] exp(DIR * 2*pi*i * n*t / N)      (DIR = -1 forward)
// One stage of radix R on the current length n_s = N/s (s = product of the
// radices already applied, m = n_s/R):
//     a_r = x[q + s(p + r m)],   y[q + s(R p + t)] = W_N^{p t s} * DFT_R(a)_t
// Each stage loads its butterfly inputs into registers, synchronises, then
// stores its outputs in place (so one buffer suffices), and synchronises.
// Radix-2/3/4/5/8/16 butterflies run in registers; twiddles W_N^k come from a
// table computed on the host in extended precision.
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
template <typename T, int DIR> __device__ __forceinline__ void dft3(C2<T>* a) {
    const T half = (T)0.5, s3 = (T)0.86602540378443864676;   // sin(2pi/3)
    C2<T> t1 = cadd(a[1], a[2]);
    C2<T> t2 = csub(a[0], cscale(half, t1));
    C2<T> t3 = rot90<DIR>(cscale(s3, csub(a[1], a[2])));
    a[0] = cadd(a[0], t1);
    a[1] = cadd(t2, t3);
    a[2] = csub(t2, t3);
}
template <typename T, int DIR> __device__ __forceinline__ void dft5(C2<T>* a) {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;   // cos(2pi/5), cos(4pi/5)
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;    // sin(2pi/5), sin(4pi/5)
    C2<T> b1 = cadd(a[1], a[4]), b2 = cadd(a[2], a[3]);
    C2<T> d1 = csub(a[1], a[4]), d2 = csub(a[2], a[3]);
    C2<T> r1 = cadd(a[0], cadd(cscale(c1, b1), cscale(c2, b2)));
    C2<T> r2 = cadd(a[0], cadd(cscale(c2, b1), cscale(c1, b2)));
    C2<T> i1 = rot90<DIR>(cadd(cscale(s1, d1), cscale(s2, d2)));
    C2<T> i2 = rot90<DIR>(csub(cscale(s2, d1), cscale(s1, d2)));
    a[0] = cadd(a[0], cadd(b1, b2));
    a[1] = cadd(r1, i1); a[4] = csub(r1, i1);
    a[2] = cadd(r2, i2); a[3] = csub(r2, i2);
}
template <typename T, int R, int DIR> __device__ __forceinline__ void dftR(C2<T>* a) {
    if (R == 2) dft2<T, DIR>(a);
    else if (R == 3) dft3<T, DIR>(a);
    else if (R == 4) dft4<T, DIR>(a);
    else if (R == 5) dft5<T, DIR>(a);
    else if (R == 8) dft8<T, DIR>(a);
    else if (R == 16) dft16<T, DIR>(a);
}

// Plan of one axis length: radices applied in order, twiddle table W_N^k.
struct FftPlan {
    int n;
    int nst;
    int radix[12];
    const void* tw;   // C2<T>[n]: exp(-2 pi i k/n), in the pass precision
};

// Element n of a column at n (PAD = 0) or n + n/16 (PAD = 1: one pad slot
// per 16 elements breaks the stride-R bank conflicts of contiguous columns).
template <int PAD> __device__ __forceinline__ int padi(int n) { return PAD ? n + (n >> 4) : n; }
__host__ __device__ inline int padded_len(int n) { return n + (n >> 4); }

// One Stockham stage over all columns, power-of-two geometry: every index is
// a shift or a mask.  ln = log2 N, lncol = log2 ncol, ls = log2 s.
// EPT = elements per thread (compile time); a thread owns ceil(EPT/R)
// butterflies.  COLFAST: consecutive threads take consecutive columns
// (columns adjacent in memory), else consecutive butterflies of a column.
template <typename T, int R, int LR, int DIR, int EPT, bool COLFAST, int PAD>
__device__ __forceinline__ void stage_p2(C2<T>* buf, int es, int cs, int ln, int ncol, int lncol, int ls,
                                         const C2<T>* __restrict__ tw) {
    constexpr int BPT = (EPT + R - 1) / R;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int lnbf = ln - LR;          // log2(N/R)
    const int lm = lnbf - ls;          // log2(m)
    const int nb = ncol << lnbf;
    const int smask = (1 << ls) - 1;
    C2<T> a[BPT][R];
#pragma unroll
    for (int u = 0; u < BPT; u++) {
        const int b = tid + u * nthr;
        if (b < nb) {
            int col, beta;
            if (COLFAST) { col = b & ((1 << lncol) - 1); beta = b >> lncol; }
            else         { beta = b & ((1 << lnbf) - 1); col = b >> lnbf; }
            const int p = beta >> ls, q = beta & smask;
            const C2<T>* base = buf + (size_t)col * cs;
            const int i0 = q + (p << ls);
#pragma unroll
            for (int r = 0; r < R; r++) a[u][r] = base[padi<PAD>(i0 + (r << (ls + lm))) * es];
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < BPT; u++) {
        const int b = tid + u * nthr;
        if (b < nb) {
            int col, beta;
            if (COLFAST) { col = b & ((1 << lncol) - 1); beta = b >> lncol; }
            else         { beta = b & ((1 << lnbf) - 1); col = b >> lnbf; }
            const int p = beta >> ls, q = beta & smask;
            dftR<T, R, DIR>(a[u]);
            C2<T>* base = buf + (size_t)col * cs;
            const int o0 = q + ((R * p) << ls);
            base[padi<PAD>(o0) * es] = a[u][0];
#pragma unroll
            for (int t = 1; t < R; t++) {
                C2<T> w = tw[(p * t) << ls];
                if (DIR > 0) w.y = -w.y;
                base[padi<PAD>(o0 + (t << ls)) * es] = (p == 0) ? a[u][t] : cmul(a[u][t], w);
            }
        }
    }
    __syncthreads();
}

// Full-radix stages (RF = 16 in FP32, 8 in FP64: the FP64 radix-16
// butterfly does not fit the register budget) in a loop with one code copy,
// then at most one stage each of radix 8, 4, 2.  Power-of-two lengths only:
// a general-length path in the same kernel costs registers (and spills) even
// when it never runs.
template <typename T> struct FullRadix { static constexpr int R = 16; static constexpr int LR = 4; };
template <> struct FullRadix<double> { static constexpr int R = 8; static constexpr int LR = 3; };

__host__ __device__ inline int ilog2(int n) { int l = 0; while ((1 << l) < n) l++; return l; }

template <typename T, int DIR, int EPT, bool COLFAST, int PAD>
__device__ __forceinline__ void fft_run(C2<T>* buf, int es, int cs, int ncol, const FftPlan& pl) {
    constexpr int RF = FullRadix<T>::R, LRF = FullRadix<T>::LR;
    const C2<T>* tw = (const C2<T>*)pl.tw;
    asm volatile("" : "+l"(tw));   // keep twiddle loads inside the caller's channel loop
    const int n = pl.n;
    {
        const int ln = ilog2(n), lncol = ilog2(ncol);   // COLFAST requires a power-of-two ncol
        int ls = 0, rest = ln;
#pragma unroll 1
        while (rest >= LRF) { stage_p2<T, RF, LRF, DIR, EPT, COLFAST, PAD>(buf, es, cs, ln, ncol, lncol, ls, tw); ls += LRF; rest -= LRF; }
        if (RF > 8 && rest >= 3) { stage_p2<T, 8, 3, DIR, EPT, COLFAST, PAD>(buf, es, cs, ln, ncol, lncol, ls, tw); ls += 3; rest -= 3; }
        if (rest >= 2) { stage_p2<T, 4, 2, DIR, EPT, COLFAST, PAD>(buf, es, cs, ln, ncol, lncol, ls, tw); ls += 2; rest -= 2; }
        if (rest >= 1) { stage_p2<T, 2, 1, DIR, EPT, COLFAST, PAD>(buf, es, cs, ln, ncol, lncol, ls, tw); }
        return;
    }
}

// Host check mirroring fft_run: power-of-two lengths, 2 <= n <= 1024.
inline bool fft_supported(int n, int RF) {
    (void)RF;
    return n >= 2 && n <= 1024 && (n & (n - 1)) == 0;
}

}  // namespace spk
