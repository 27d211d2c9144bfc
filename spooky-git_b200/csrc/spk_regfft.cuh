// spk_regfft.cuh -- register-resident FFT of compile-time length for sm_100a.
//
// A length-N transform, N = 2^k (2..1024) or N = 3*2^k (6..768), is split
// over TPC = N/E cooperating threads, each holding E elements in registers:
//   N = 2^k:   E = 16 (FP32) or 8 (FP64) (N when smaller); stages of the
//              full radix E, then one smaller power-of-two radix;
//   N = 3*2^k: E = 12 (6 for N = 6); a radix-3 stage, radix-4 stages, and
//              one radix-2 stage when k is odd.
// Decimation in frequency, written from the DFT definition
// X[k] = sum_n x[n] exp(DIR 2 pi i n k / N):
//
//   stage s has radix R_s; before it the sequence is split into
//   P_s = R_0...R_{s-1} groups of length M_s = N/P_s.  A butterfly (g, m),
//   m < H_s = M_s/R_s, takes a_r = z_g[m + H_s r], forms
//   y_t = W_{M_s}^{m t} sum_r a_r w_R^{r t} and hands it on as element m of
//   group g + P_s t.  After the last stage group g holds X[g].
//
// The first stage reads its inputs through the caller's functor `load(n)`
// (shared-memory tile, paired half spectra, ...), stages meet through one
// shared-memory exchange each (so a 256-point FP32 transform makes exactly
// one), and the last stage hands X[k] to the caller's `store(k, v)` from
// registers (a global store, a shared-memory store, a product).  Twiddles
// come from per-stage shared-memory tables of the pass precision, laid out
// so that the threads of one transform read consecutive words.  Every
// stage constant is known at compile time (H_s is a power of two, so the
// divisions by it are shifts).
#pragma once
#include "spk_fft.cuh"

namespace spk {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }
__host__ __device__ constexpr bool is_pow2c(int n) { return n > 0 && (n & (n - 1)) == 0; }
// Lengths the register-resident transforms cover.
__host__ __device__ constexpr bool regfft_length_ok(int n) {
    return n >= 2 && n <= 1024 && (is_pow2c(n) || (n >= 6 && n % 3 == 0 && is_pow2c(n / 3)));
}

template <typename T, int N>
struct RegFft {
    static_assert(regfft_length_ok(N), "transform length must be 2^k (2..1024) or 3*2^k (6..768)");
    static constexpr bool P2 = is_pow2c(N);
    static constexpr int LRF = sizeof(T) == 4 ? 4 : 3;                 // full radix 16 (FP32) / 8 (FP64)
    static constexpr int LN2 = P2 ? ilog2c(N) : ilog2c(N / 3);         // the power-of-two part
    static constexpr int E = P2 ? (LN2 < LRF ? N : (1 << LRF)) : (N < 12 ? N : 12);
    static constexpr int TPC = N / E;                                 // threads per transform
    static constexpr int LTPC = ilog2c(TPC);
    static constexpr int NFULL = P2 ? LN2 / LRF : 0;
    static constexpr int NS = P2 ? (LN2 + LRF - 1) / LRF : 1 + LN2 / 2 + LN2 % 2;   // stages
    static constexpr int radix(int s) {
        return P2 ? (s < NFULL ? (1 << LRF) : (1 << (LN2 - NFULL * LRF))) : (s == 0 ? 3 : (s <= LN2 / 2 ? 4 : 2));
    }
    static constexpr int P(int s) { return s == 0 ? 1 : P(s - 1) * radix(s - 1); }
    static constexpr int M(int s) { return N / P(s); }
    static constexpr int H(int s) { return M(s) / radix(s); }
    // Twiddle tables: stage s (H_s > 1) keeps W_N^{m t P_s} at tbase(s) + t*H_s + m,
    // M_s entries, so that consecutive m (consecutive threads) read consecutive words.
    static constexpr int tbase(int s) { return s == 0 ? 0 : tbase(s - 1) + M(s - 1); }
    static constexpr int TWN = NS > 1 ? tbase(NS - 1) : 1;             // entries over all stages
};

template <typename T, int DIR> __device__ __forceinline__ void dft3(C2<T>* a) {
    const T half = (T)0.5, s3 = (T)0.86602540378443864676;   // sin(2 pi / 3)
    const C2<T> t1 = cadd(a[1], a[2]);
    const C2<T> t2 = csub(a[0], cscale(half, t1));
    const C2<T> t3 = rot90<DIR>(cscale(s3, csub(a[1], a[2])));
    a[0] = cadd(a[0], t1);
    a[1] = cadd(t2, t3);
    a[2] = csub(t2, t3);
}

template <typename T, int R, int DIR> __device__ __forceinline__ void dft_r(C2<T>* a) {
    if constexpr (R == 2) dft2<T, DIR>(a);
    else if constexpr (R == 3) dft3<T, DIR>(a);
    else if constexpr (R == 4) dft4<T, DIR>(a);
    else if constexpr (R == 8) dft8<T, DIR>(a);
    else if constexpr (R == 16) dft16<T, DIR>(a);
}

// Fill the per-stage twiddle tables from the table W_N^j (all threads call).
template <typename T, int N>
__device__ __forceinline__ void regfft_fill_twiddles(C2<T>* tws, const C2<T>* twg, int tid, int nthr) {
    using F = RegFft<T, N>;
    for (int i = tid; i < F::TWN; i += nthr) {
        int h = 1, pp = 1, tb = 0;
#pragma unroll
        for (int k = 0; k + 1 < F::NS; k++)
            if (i >= F::tbase(k)) { h = F::H(k); pp = F::P(k); tb = F::tbase(k); }
        const int e = i - tb;
        const int t = e / h, m = e - t * h;
        tws[i] = twg[m * t * pp];
    }
}

// Table entry j (W_N^k for some k, DIR = -1) or its conjugate (DIR = +1).
template <typename T, int DIR> __device__ __forceinline__ C2<T> twd(const C2<T>* tw, int j) {
    C2<T> w = tw[j];
    if (DIR > 0) w.y = -w.y;
    return w;
}

// Run stage S (butterflies of this thread, q = sub-index within the
// transform) on registers a[E] whose legs are already loaded; apply the
// twiddles from the per-stage tables.  Leg t of butterfly u ends in a[u*R + t].
template <typename T, int N, int DIR, int S>
__device__ __forceinline__ void regfft_stage_math(C2<T>* a, int q, const C2<T>* tw) {
    using F = RegFft<T, N>;
    constexpr int R = F::radix(S), H = F::H(S);
    constexpr int BPT = F::E / R;
#pragma unroll
    for (int u = 0; u < BPT; u++) {
        dft_r<T, R, DIR>(a + u * R);
        if constexpr (H > 1) {
            const unsigned beta = (unsigned)q + (unsigned)(u * F::TPC);   // unsigned: % and / by H are masks and shifts
            const int m = (int)(beta % (unsigned)H);
            const C2<T>* tws = tw + F::tbase(S) + m;
#pragma unroll
            for (int t = 1; t < R; t++) a[u * R + t] = cmul(a[u * R + t], twd<T, DIR>(tws, t * H));
        }
    }
}

// Element index (in the linear exchange layout g*M + position) of leg r of
// butterfly u at stage S.
template <typename T, int N, int S>
__device__ __forceinline__ int regfft_in_index(int q, int u, int r) {
    using F = RegFft<T, N>;
    constexpr int H = F::H(S), M = F::M(S);
    const unsigned beta = (unsigned)q + (unsigned)(u * F::TPC);
    const int m = (int)(beta % (unsigned)H), g = (int)(beta / (unsigned)H);
    return g * M + m + r * H;
}
// Linear exchange index where output t of butterfly u of stage S goes
// (element m of group g + P t, in a layout of groups of length H).
template <typename T, int N, int S>
__device__ __forceinline__ int regfft_out_index(int q, int u, int t) {
    using F = RegFft<T, N>;
    constexpr int H = F::H(S), P = F::P(S);
    const unsigned beta = (unsigned)q + (unsigned)(u * F::TPC);
    const int m = (int)(beta % (unsigned)H), g = (int)(beta / (unsigned)H);
    return (g + P * t) * H + m;
}

// One exchange between stages S and S+1.  xaddr(L) is the shared-memory slot
// of exchange element L (the caller picks layout and padding).  Every thread
// of the CTA must call it: it starts with a barrier (earlier reads of the
// buffer, including a previous tile's, are complete) and ends with one (the
// writes are visible).
// act = false: a thread with no transform to run (it must be false for a
// whole warp at a time) only takes part in the barriers, which stay at the
// same instructions for every warp of the CTA.
// XB: 0, or the pad block of the caller's layout: xaddr(L) is a fixed base
// plus L + L/XB (XB a power of two).  Where the legs of a butterfly step
// through L by a multiple of XB, or stay inside one aligned block of XB,
// their padded positions are the first leg's plus a compile-time offset,
// and the exchange addresses them from one pointer.
template <typename T, int N, int DIR, int S, int XB = 0, typename XA>
__device__ __forceinline__ void regfft_exchange(C2<T>* a, int q, XA xaddr, bool act = true) {
    using F = RegFft<T, N>;
    constexpr int R = F::radix(S);
    constexpr int BPT = F::E / R;
    constexpr int XBD = XB > 0 ? XB : 1;   // a nonzero divisor for the XB = 0 branches
    __syncthreads();   // earlier readers of the exchange buffer are done
    if (act) {
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            // leg t of the writes is at L0 + P H t
            constexpr int DL = F::P(S) * F::H(S);
            if constexpr (XB > 0 && DL % XBD == 0) {
                C2<T>* p0 = xaddr(regfft_out_index<T, N, S>(q, u, 0));
#pragma unroll
                for (int t = 0; t < R; t++) p0[t * (DL + DL / XBD)] = a[u * R + t];
            } else {
#pragma unroll
                for (int t = 0; t < R; t++) *xaddr(regfft_out_index<T, N, S>(q, u, t)) = a[u * R + t];
            }
        }
    }
    __syncthreads();
    constexpr int R1 = F::radix(S + 1);
    constexpr int BPT1 = F::E / R1;
    constexpr int H1 = F::H(S + 1);
    if (act) {
#pragma unroll
        for (int u = 0; u < BPT1; u++) {
            // leg r of the reads is at L0 + H1 r; with H1 = 1 the legs lie in one
            // aligned block of XB when R1 is a power of two up to XB
            if constexpr (XB > 0 && H1 % XBD == 0) {
                const C2<T>* p0 = xaddr(regfft_in_index<T, N, S + 1>(q, u, 0));
#pragma unroll
                for (int r = 0; r < R1; r++) a[u * R1 + r] = p0[r * (H1 + H1 / XBD)];
            } else if constexpr (XB > 0 && H1 == 1 && is_pow2c(R1) && R1 <= XB) {
                const C2<T>* p0 = xaddr(regfft_in_index<T, N, S + 1>(q, u, 0));
#pragma unroll
                for (int r = 0; r < R1; r++) a[u * R1 + r] = p0[r];
            } else {
#pragma unroll
                for (int r = 0; r < R1; r++) a[u * R1 + r] = *xaddr(regfft_in_index<T, N, S + 1>(q, u, r));
            }
        }
    }
}

// FS: barrier before the last stage's stores (when store() writes into the
// exchange buffer that the last exchange just read).  act: as for
// regfft_exchange (no math, no stores, the same barriers).
template <typename T, int N, int DIR, int S, bool FS, int XB, typename XA, typename ST>
__device__ __forceinline__ void regfft_from(C2<T>* a, int q, const C2<T>* tw, XA xaddr, ST store, bool act = true) {
    using F = RegFft<T, N>;
    if (act) regfft_stage_math<T, N, DIR, S>(a, q, tw);
    if constexpr (S + 1 < F::NS) {
        regfft_exchange<T, N, DIR, S, XB>(a, q, xaddr, act);
        regfft_from<T, N, DIR, S + 1, FS, XB>(a, q, tw, xaddr, store, act);
    } else {
        if constexpr (FS && S > 0) __syncthreads();
        constexpr int R = F::radix(S), P = F::P(S);
        constexpr int BPT = F::E / R;
        if (!act) return;
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int g = q + u * F::TPC;   // last stage: H = 1, beta = g
#pragma unroll
            for (int t = 0; t < R; t++) store(g + P * t, a[u * R + t]);
        }
    }
}

// Bit u*R + t set where pred(k) holds for the output k that thread q hands
// to store() as its (u, t)-th call of the last stage (the order of
// regfft_from's stores), so that a caller can test a per-output condition
// from one register.
template <typename T, int N, typename PR>
__device__ __forceinline__ uint32_t regfft_store_mask(int q, PR pred) {
    using F = RegFft<T, N>;
    static_assert(F::E <= 32, "one bit per element");
    constexpr int S = F::NS - 1, R = F::radix(S), P = F::P(S);
    constexpr int BPT = F::E / R;
    uint32_t m = 0;
#pragma unroll
    for (int u = 0; u < BPT; u++)
#pragma unroll
        for (int t = 0; t < R; t++)
            if (pred((q + u * F::TPC) + P * t)) m |= 1u << (u * R + t);
    return m;
}

// Bit u*R + r set where pred(n) holds for the input n that thread q reads
// as its (u, r)-th call of load() in regfft_load.
template <typename T, int N, typename PR>
__device__ __forceinline__ uint32_t regfft_load_mask(int q, PR pred) {
    using F = RegFft<T, N>;
    static_assert(F::E <= 32, "one bit per element");
    constexpr int R = F::radix(0);
    constexpr int BPT = F::E / R;
    uint32_t m = 0;
#pragma unroll
    for (int u = 0; u < BPT; u++)
#pragma unroll
        for (int r = 0; r < R; r++)
            if (pred(regfft_in_index<T, N, 0>(q, u, r))) m |= 1u << (u * R + r);
    return m;
}

// Load the first-stage legs through load(n).
template <typename T, int N, int DIR, typename LD>
__device__ __forceinline__ void regfft_load(C2<T>* a, int q, LD load) {
    using F = RegFft<T, N>;
    constexpr int R = F::radix(0);
    constexpr int BPT = F::E / R;
#pragma unroll
    for (int u = 0; u < BPT; u++)
#pragma unroll
        for (int r = 0; r < R; r++) a[u * R + r] = load(regfft_in_index<T, N, 0>(q, u, r));
}

// XB: see regfft_exchange (0, or the pad block of xaddr's layout).
template <typename T, int N, int DIR, bool FS = false, int XB = 0, typename XA, typename ST>
__device__ __forceinline__ void regfft_run(C2<T>* a, int q, const C2<T>* tw, XA xaddr, ST store, bool act = true) {
    regfft_from<T, N, DIR, 0, FS, XB>(a, q, tw, xaddr, store, act);
}

// Host mirror of the geometry.
struct RegFftGeom { int E, TPC; };
inline RegFftGeom regfft_geom(int n, bool fp32) {
    RegFftGeom g;
    if (is_pow2c(n)) {
        const int lrf = fp32 ? 4 : 3, ln = ilog2c(n);
        g.E = ln < lrf ? n : (1 << lrf);
    } else {
        g.E = n < 12 ? n : 12;
    }
    g.TPC = n / g.E;
    return g;
}

}  // namespace spk
