// spk_regfft.cuh -- register-resident FFT of compile-time length for sm_100a.
//
// A length N = 2^LN transform is split over TPC = N/E cooperating threads,
// each holding E = 2^LE elements in registers (E = 16 in FP32, 8 in FP64;
// E = N when N is smaller).  Decimation in frequency, written from the DFT
// definition X[k] = sum_n x[n] exp(DIR 2 pi i n k / N):
//
//   stage s has radix R_s = 2^lr(s); before it the sequence is split into
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
// so that the threads of one transform read consecutive words.
#pragma once
#include "spk_fft.cuh"

namespace spk {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

template <typename T, int LN>
struct RegFft {
    static constexpr int LRF = sizeof(T) == 4 ? 4 : 3;       // full radix 16 (FP32) / 8 (FP64)
    static constexpr int N = 1 << LN;
    static constexpr int LE = LN < LRF ? LN : LRF;
    static constexpr int E = 1 << LE;                        // elements per thread
    static constexpr int LTPC = LN - LE;
    static constexpr int TPC = 1 << LTPC;                    // threads per transform
    static constexpr int NFULL = LN / LRF;
    static constexpr int NS = (LN + LRF - 1) / LRF;          // stages
    static constexpr int lr(int s) { return s < NFULL ? LRF : LN - NFULL * LRF; }
    static constexpr int ls(int s) { return s == 0 ? 0 : ls(s - 1) + lr(s - 1); }   // log2 P_s
    // Twiddle tables: stage s (H_s > 1) keeps W_N^{(m t) P_s} at tbase(s) + t*H_s + m,
    // M_s entries, so that consecutive m (consecutive threads) read consecutive words.
    static constexpr int tbase(int s) { return s == 0 ? 0 : tbase(s - 1) + (N >> ls(s - 1)); }
    static constexpr int TWN = NS > 1 ? tbase(NS - 1) : 1;   // entries over all stages
};

// Fill the per-stage twiddle tables from the table W_N^j (all threads call).
template <typename T, int LN>
__device__ __forceinline__ void regfft_fill_twiddles(C2<T>* tws, const C2<T>* twg, int tid, int nthr) {
    using F = RegFft<T, LN>;
    for (int i = tid; i < F::TWN; i += nthr) {
        int s = 0;
        while (s + 1 < F::NS && i >= F::tbase(s + 1)) s++;
        const int lh = LN - F::ls(s) - F::lr(s);
        const int e = i - F::tbase(s);
        const int t = e >> lh, m = e & ((1 << lh) - 1);
        tws[i] = twg[(m * t) << F::ls(s)];
    }
}

template <typename T, int R, int DIR> __device__ __forceinline__ void dft_pow2(C2<T>* a) {
    if constexpr (R == 2) dft2<T, DIR>(a);
    else if constexpr (R == 4) dft4<T, DIR>(a);
    else if constexpr (R == 8) dft8<T, DIR>(a);
    else if constexpr (R == 16) dft16<T, DIR>(a);
}

// Table entry j (W_N^k for some k, DIR = -1) or its conjugate (DIR = +1).
template <typename T, int DIR> __device__ __forceinline__ C2<T> twd(const C2<T>* tw, int j) {
    C2<T> w = tw[j];
    if (DIR > 0) w.y = -w.y;
    return w;
}

// Run stage S (butterflies of this thread, q = sub-index within the
// transform) on registers a[E] whose legs are already loaded; apply the
// twiddles from the per-stage tables (regfft_fill_twiddles).  Leg t of
// butterfly u ends in a[u*R + t].
template <typename T, int LN, int DIR, int S>
__device__ __forceinline__ void regfft_stage_math(C2<T>* a, int q, const C2<T>* tw) {
    using F = RegFft<T, LN>;
    constexpr int LR = F::lr(S), R = 1 << LR;
    constexpr int LP = F::ls(S);
    constexpr int LM = LN - LP, LH = LM - LR;
    constexpr int BPT = F::E >> LR;
#pragma unroll
    for (int u = 0; u < BPT; u++) {
        dft_pow2<T, R, DIR>(a + u * R);
        if constexpr (LH > 0) {
            const int beta = q + (u << F::LTPC);
            const int m = beta & ((1 << LH) - 1);
            const C2<T>* tws = tw + F::tbase(S) + m;
#pragma unroll
            for (int t = 1; t < R; t++) a[u * R + t] = cmul(a[u * R + t], twd<T, DIR>(tws, t << LH));
        }
    }
}

// Element index (in the linear exchange layout g*M + position) of leg r of
// butterfly u at stage S.
template <typename T, int LN, int S>
__device__ __forceinline__ int regfft_in_index(int q, int u, int r) {
    using F = RegFft<T, LN>;
    constexpr int LR = F::lr(S), LP = F::ls(S);
    constexpr int LM = LN - LP, LH = LM - LR;
    const int beta = q + (u << F::LTPC);
    const int m = beta & ((1 << LH) - 1), g = beta >> LH;
    return (g << LM) + m + (r << LH);
}
// Linear exchange index where output t of butterfly u of stage S goes
// (element m of group g + P t, in a layout of groups of length H).
template <typename T, int LN, int S>
__device__ __forceinline__ int regfft_out_index(int q, int u, int t) {
    using F = RegFft<T, LN>;
    constexpr int LR = F::lr(S), LP = F::ls(S);
    constexpr int LM = LN - LP, LH = LM - LR;
    const int beta = q + (u << F::LTPC);
    const int m = beta & ((1 << LH) - 1), g = beta >> LH;
    return ((g + (t << LP)) << LH) + m;
}

// Full transform.  load(n) gives input n; xaddr(L) is the shared-memory slot
// of exchange element L (the caller picks layout and padding); store(k, v)
// receives X[k]; tw holds the per-stage twiddle tables.  Every thread of
// the CTA must call it: each exchange
// starts with a barrier (earlier reads of the buffer, including a previous
// tile's, are complete) and ends with one (the writes are visible).
template <typename T, int LN, int DIR, int S, typename XA>
__device__ __forceinline__ void regfft_exchange(C2<T>* a, int q, XA xaddr) {
    using F = RegFft<T, LN>;
    constexpr int R = 1 << F::lr(S);
    constexpr int BPT = F::E / R;
    __syncthreads();   // earlier readers of the exchange buffer are done
#pragma unroll
    for (int u = 0; u < BPT; u++)
#pragma unroll
        for (int t = 0; t < R; t++) *xaddr(regfft_out_index<T, LN, S>(q, u, t)) = a[u * R + t];
    __syncthreads();
    constexpr int R1 = 1 << F::lr(S + 1);
    constexpr int BPT1 = F::E / R1;
#pragma unroll
    for (int u = 0; u < BPT1; u++)
#pragma unroll
        for (int r = 0; r < R1; r++) a[u * R1 + r] = *xaddr(regfft_in_index<T, LN, S + 1>(q, u, r));
}

// FS: barrier before the last stage's stores (when store() writes into the
// exchange buffer that the last exchange just read).
template <typename T, int LN, int DIR, int S, bool FS, typename XA, typename ST>
__device__ __forceinline__ void regfft_from(C2<T>* a, int q, const C2<T>* tw, XA xaddr, ST store) {
    using F = RegFft<T, LN>;
    regfft_stage_math<T, LN, DIR, S>(a, q, tw);
    if constexpr (S + 1 < F::NS) {
        regfft_exchange<T, LN, DIR, S>(a, q, xaddr);
        regfft_from<T, LN, DIR, S + 1, FS>(a, q, tw, xaddr, store);
    } else {
        if constexpr (FS && S > 0) __syncthreads();
        constexpr int LR = F::lr(S), R = 1 << LR, LP = F::ls(S);
        constexpr int BPT = F::E / R;
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int g = q + (u << F::LTPC);   // last stage: H = 1, beta = g
#pragma unroll
            for (int t = 0; t < R; t++) store(g + (t << LP), a[u * R + t]);
        }
    }
}

// Load the first-stage legs through load(n), then transform.
template <typename T, int LN, int DIR, typename LD>
__device__ __forceinline__ void regfft_load(C2<T>* a, int q, LD load) {
    using F = RegFft<T, LN>;
    constexpr int R = 1 << F::lr(0);
    constexpr int BPT = F::E / R;
#pragma unroll
    for (int u = 0; u < BPT; u++)
#pragma unroll
        for (int r = 0; r < R; r++) a[u * R + r] = load(regfft_in_index<T, LN, 0>(q, u, r));
}

template <typename T, int LN, int DIR, bool FS = false, typename XA, typename ST>
__device__ __forceinline__ void regfft_run(C2<T>* a, int q, const C2<T>* tw, XA xaddr, ST store) {
    regfft_from<T, LN, DIR, 0, FS>(a, q, tw, xaddr, store);
}

// Host mirror of the geometry.
struct RegFftGeom { int E, TPC, NS; };
inline RegFftGeom regfft_geom(int n, bool fp32) {
    const int lrf = fp32 ? 4 : 3;
    int ln = ilog2(n);
    const int le = ln < lrf ? ln : lrf;
    RegFftGeom g;
    g.E = 1 << le;
    g.TPC = 1 << (ln - le);
    g.NS = (ln + lrf - 1) / lrf;
    return g;
}

}  // namespace spk
