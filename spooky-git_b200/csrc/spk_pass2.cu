// spk_pass2.cu -- strided-axis FFT pass on the register-resident FFT.
//
// Tile = one channel, one outer index, KT consecutive k columns, all N
// positions along the axis ([N][KT] in shared memory, the TMA box layout).
// A persistent CTA keeps nst tiles in flight with cp.async.bulk.tensor loads
// completing on per-stage mbarriers (bounded waits).  For each tile, thread
// (column c, sub-index q) reads its first-stage legs straight from the
// stage buffer -- converting the FP64 state, applying the 1/N^3 scale of
// scaleKernel (cufft_routines.cu:23-39) and the i*k derivative of Gradient
// (cuda_kernels_generic.cu:249-260) on the way -- releases the stage to the
// next load, runs the transform in registers with one shared-memory
// exchange per further stage, and stores X[k] from registers to the pass
// buffer (kept ky rows only in the y-forward pass).
#include "spk_regfft.cuh"
#include "spk_closure.cuh"
#include "spk_closure3.cuh"

namespace spk {

// Tile width of the strided-axis pass: KT columns x TPC threads = 256
// threads (KT <= 64); an FP64 input tile in the FP32 form (CONV) is half as
// wide so that one pipeline stage stays at 32 KB.
//
// Short axes (N < 64) take the tile no wider than the kz columns of a cubic
// box, N/2 + 1 rounded up to a power of two, and at least one warp per CTA:
// a 64-column tile on a 16^3 box would transform 55 columns of padding.
__host__ __device__ constexpr int pow2_ceil(int n) { return n <= 1 ? 1 : 2 * pow2_ceil((n + 1) / 2); }
template <typename T, int N, bool CONV>
__host__ __device__ constexpr int axis_kt_base() {
    constexpr int tpc = RegFft<T, N>::TPC;
    constexpr int full = (256 / tpc) > 64 ? 64 : (256 / tpc);
    constexpr int cols = pow2_ceil(N / 2 + 1) > 32 / tpc ? pow2_ceil(N / 2 + 1) : 32 / tpc;
    constexpr int kt = (N < 64 && cols < full) ? cols : full;
    return (CONV && kt == full && kt > 2) ? kt / 2 : (kt < 2 ? 2 : kt);
}
// Short axes (N <= 64) also come in half-width tiles (KTD = 2), an
// autotuner choice: a 64^3 box has 33 kz columns (21 below the 2/3 cut-off)
// in a 64-column tile.  The half tile keeps at least one warp per CTA.
template <typename T, int N, bool CONV>
__host__ __device__ constexpr bool axis_half_ok() {
    return N <= 64 && axis_kt_base<T, N, CONV>() / 2 >= 2 &&
           (axis_kt_base<T, N, CONV>() / 2) * RegFft<T, N>::TPC >= 32;
}
template <typename T, int N, bool CONV, int KTD = 1>
__host__ __device__ constexpr int axis_kt() {
    return axis_kt_base<T, N, CONV>() / KTD;
}

// CTAs per SM the strided-axis pass is compiled for.  FP64 transforms of
// up to 256 points hold at most 8 elements per thread and fit 80 registers
// with little spilling, so three CTAs (one pipeline stage each) keep more
// warps resident (256^3 plain form: 6.00 -> 5.75 ms per step).  The FP32
// form's 16 elements per thread, and the longer FP64 transforms, spill at 80
// registers and keep two CTAs (512^3 plain form: 59.8 ms with two, 69.9 ms
// with three).
template <typename T, int N> __host__ __device__ constexpr int axis_minb() {
    return (sizeof(T) == 8 && N <= 256 && RegFft<T, N>::E <= 8) ? 3 : 2;
}

// DEF: the x inverse of RK3 stage 1 or 2 with deferred masked modes (its own
// instantiation, so that the other passes keep their registers).  KTD: tile
// width divisor (1, or 2 for the half tiles of short axes).
template <typename T, int N, int DIR, bool CONV, bool DEF, int KTD>
__global__ void __launch_bounds__(256, axis_minb<T, N>()) k_axis2(const __grid_constant__ AxisArgs a) {
    using F = RegFft<T, N>;
    constexpr int KT = axis_kt<T, N, CONV, KTD>(), LKT = ilog2c(KT);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (a.gate && a.gate_stage > a.gate->s_rkl) return;
    const int NST = a.nst;
    const int tid = threadIdx.x;
    const int c = tid & (KT - 1), q = tid >> LKT;
    const int nouter = a.axis == 0 ? a.g.ny : a.g.nx;
    // a trimmed pass whose boxes all have no masked content walks only the
    // tiles it keeps (every CTA reads the same flags)
    bool all_clear = a.trim != 0;
    for (int b = 0; all_clear && b < a.nb; b++) all_clear = !a.scs[b].masked_live;
    const bool ctile = a.tr_always || all_clear;
    const bool couter = ctile && (a.trim == 1 || a.tr_always);
    const int nkb = ctile ? a.tr_nkb : (a.kcols + KT - 1) / KT;
    const int nouter_e = couter ? a.tr_nouter : nouter;
    const FastDiv fdj = ctile ? a.tr_fd_job : a.fd_job, fdb = ctile ? a.tr_fd_box : a.fd_box;
    const FastDiv fdk = ctile ? a.tr_fd_kb : a.fd_kb;
    const int per_box = nouter_e * nkb;
    const int per_job = a.nb * per_box;
    const int total = a.njobs * per_job;   // tile t = ((job * nb + box) * nouter + o) * nkb + kb
    constexpr size_t in_elem = CONV ? sizeof(double2) : sizeof(C2<T>);
    constexpr size_t stage_bytes = ((size_t)N * KT * in_elem + 127) & ~(size_t)127;
    unsigned char* sbase = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase);
    unsigned char* stages = sbase + 128;
    C2<T>* xbuf = reinterpret_cast<C2<T>*>(stages + (size_t)NST * stage_bytes);
    C2<T>* tw = xbuf + (size_t)N * KT;
    T* kax = reinterpret_cast<T*>(tw + F::TWN);                      // wavenumbers along the axis
    unsigned char* keep = reinterpret_cast<unsigned char*>(kax + N);  // row mask factor != 0
    unsigned char* okeep = keep + N;                                  // outer-index mask factor != 0
    const int stride = a.axis == 0 ? a.g.ny * a.g.nzs : a.g.nzs;
    constexpr uint32_t tile_bytes = (uint32_t)((size_t)N * KT * in_elem);
    const uint32_t box_bytes = tile_bytes / (uint32_t)(N / a.box_rows);

    // tiles that a trimmed pass skips (uniform: every thread decides alike)
    auto trimmed = [&](int box, int o, int kb) -> bool {
        if (!a.trim || a.scs[box].masked_live) return false;
        return kb * KT >= a.g.kz_keep || (a.trim == 1 && !okeep[o]);
    };
    auto issue = [&](int t, int s) {
        const int jb = (int)fdj.div((unsigned)t);
        const int rb = t - jb * per_job;
        const int box = (int)fdb.div((unsigned)rb);
        const int rem = rb - box * per_box;
        const int oe = (int)fdk.div((unsigned)rem), kb = rem - oe * nkb;
        const int o = couter ? a.tr_outer[oe] : oe;
        const AxisJob& jo = a.job[jb];
        const int ch = jo.ch + box * a.in_box_ch;
        unsigned char* dst = stages + (size_t)s * stage_bytes;
        if ((a.outer_filter && !okeep[o]) || trimmed(box, o, kb)) {   // skipped tile: complete the phase with no bytes
            mbar_expect_tx(&bar[s], 0);
            return;
        }
        mbar_expect_tx(&bar[s], tile_bytes);
        for (int b = 0; b < N / a.box_rows; b++) {
            if (a.axis == 0) tma_load_4d(dst + (size_t)b * box_bytes, &jo.tm, &bar[s], 2 * kb * KT, o, b * a.box_rows, ch);
            else             tma_load_4d(dst + (size_t)b * box_bytes, &jo.tm, &bar[s], 2 * kb * KT, b * a.box_rows, o, ch);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < NST; s++) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    {
        const C2<T>* twg = (const C2<T>*)a.plan.tw;
        const double* kg = a.axis == 0 ? a.g.kx : a.g.ky;
        const double* mg = a.axis == 0 ? a.g.mx : a.g.my;
        regfft_fill_twiddles<T, N>(tw, twg, tid, blockDim.x);
        for (int i = tid; i < N; i += blockDim.x) {
            kax[i] = (T)kg[i];
            keep[i] = mg[i] != 0.0;
        }
        const double* og = a.axis == 0 ? a.g.my : a.g.mx;   // mask factor of the outer index
        for (int i = tid; i < nouter; i += blockDim.x) okeep[i] = og[i] != 0.0;
    }
    __syncthreads();
    // The kept rows among this thread's outputs (forward passes: one bit per
    // store of the last stage, the row filter) or inputs (inverse passes: one
    // bit per load of the first stage, the zero rows of the trimmed y
    // inverse), and load paths with the per-tile flags off the element loop:
    // in the forward passes, and in every pass of the two-CTA
    // instantiations.  The three-CTA (FP64) inverse passes keep the plain
    // forms, which spill less at their 80 registers.
    constexpr bool LEAN = DIR < 0 || axis_minb<T, N>() == 2;
    uint32_t keepm = ~0u;
    if constexpr (LEAN) {
        auto kept = [&](int k) { return keep[k] != 0; };
        if constexpr (DIR < 0) keepm = regfft_store_mask<T, N>(q, kept);
        else keepm = regfft_load_mask<T, N>(q, kept);
    }
    if (tid == 0)
        for (int s = 0; s < NST; s++) {
            const int t = blockIdx.x + s * gridDim.x;
            if (t < total) issue(t, s);
        }

    int i = 0;
    bool aborted = false;
    C2<T> r[F::E];
    int dbox = -1;                 // box whose deferred-mode scalars are cached
    T dnu1 = (T)0, dnu2 = (T)0;
    bool dlive = true;
    const double shx_x = DIR > 0 ? grid_shx(a.g) : 0.0;   // the shearing box's wavevector shear (0 without it)
    for (int t = blockIdx.x; t < total; t += gridDim.x, i++) {
        const int s = i % NST;
        const uint32_t par = (uint32_t)((i / NST) & 1);
        const bool ok = mbar_wait(&bar[s], par, SPK_WAIT_ITERS);
        if (__syncthreads_or(!ok)) { aborted = true; break; }
        const int jb = (int)fdj.div((unsigned)t);
        const int rb = t - jb * per_job;
        const int box = (int)fdb.div((unsigned)rb);
        const int rem = rb - box * per_box;
        const int oe = (int)fdk.div((unsigned)rem), kb = rem - oe * nkb;
        const int o = couter ? a.tr_outer[oe] : oe;
        const AxisJob& jo = a.job[jb];
        const int k0 = kb * KT;
        const int kt = min(KT, a.kcols - k0);
        const unsigned char* stg = stages + (size_t)s * stage_bytes;
        const int deriv = jo.deriv;
        const double scale = a.scale;
        // derivative along the outer index or the column, and the high-pass
        // of the closure's small scales (uniform over the CTA)
        double kout = 0.0, kcol = 0.0;
        if (deriv >= 2 || jo.hp) {
            kout = a.axis == 0 ? a.g.ky[o] : a.g.kx[o];
            kcol = a.g.kz[min(k0 + c, a.g.nzh - 1)];
        }
        // shearing box: on x lines kx(n, o) = kx[n] + shx ky[o] (0 without it;
        // only the x inverse, which reads the state, takes x derivatives)
        const double kshift = (DIR > 0 && a.axis == 0 && shx_x != 0.0) ? shx_x * a.g.ky[o] : 0.0;
        const bool skip = (a.outer_filter && !okeep[o]) || trimmed(box, o, kb);   // uniform over the CTA
        // trimmed y inverse: masked y rows were not written by the x inverse
        const bool zrows = a.trim == 2 && !skip && !a.scs[box].masked_live;
        // Deferred masked modes (x inverse of RK3 stage 1 or 2): outside the
        // 2/3 mask the state still holds the step's start value U, whereas
        // the stage reads U1 = c1(z) U or U2 = c2(z) U, z = -nu k^2 dt (the
        // recurrences of rk_value for a purely diffusive right-hand side),
        // evaluated in the pass precision.
        bool dfr = DEF && jo.defer_grp != 0;   // uniform over the CTA
        T dnu = (T)0, k2yz = (T)0;
        bool col_out = false;
        if (dfr) {
            if (box != dbox) {
                const DevScalars& bs = a.scs[box];
                dnu1 = (T)(-bs.nu * bs.dt);
                dnu2 = (T)(-bs.nu_m * bs.dt);
                dlive = bs.masked_live != 0;
                dbox = box;
            }
            dfr = dlive;   // negligible masked content: nothing to scale
        }
        if (dfr) {
            dnu = jo.defer_grp == 1 ? dnu1 : dnu2;
            const int kc = min(k0 + c, a.g.nzh - 1);
            const double kyo = a.g.ky[o], kzc = a.g.kz[kc];
            k2yz = (T)(kyo * kyo + kzc * kzc);
            col_out = !okeep[o] || k0 + c >= a.g.kz_keep;
        }
        auto deferred = [&](int n) -> T {   // factor of input row n (1 inside the mask)
            const T kxn = kax[n];
            const T z = dnu * (kxn * kxn + k2yz);
            const T c1 = (T)1 + (T)(8.0 / 15.0) * z;
            const T f = a.defer_stage == 1 ? c1 : c1 + (T)(-17.0 / 60.0) * z + (T)(5.0 / 12.0) * z * c1;
            return (col_out || !keep[n]) ? f : (T)1;
        };
        if (skip) {
        } else if (CONV && !deriv && !jo.hp && !(DEF && dfr)) {
            // FP64 input, no per-row factor
            const double2* src = reinterpret_cast<const double2*>(stg);
            regfft_load<T, N, DIR>(r, q, [&](int n) -> C2<T> {
                const double2 x = src[n * KT + c];
                return mk<T>((T)(x.x * scale), (T)(x.y * scale));
            });
        } else if constexpr (CONV) {
            const double2* src = reinterpret_cast<const double2*>(stg);
            const double* kd = a.axis == 0 ? a.g.kx : a.g.ky;   // FP64 derivative on the FP64 input
            regfft_load<T, N, DIR>(r, q, [&](int n) -> C2<T> {
                double2 x = src[n * KT + c];
                if (deriv) x = ik_mul(deriv == 1 ? kd[n] + kshift : (deriv == 2 ? kout : kcol), x);
                if (jo.hp && !(kd[n] * kd[n] + kout * kout + kcol * kcol > a.hp_k2)) x = make_double2(0.0, 0.0);
                C2<T> v = mk<T>((T)(x.x * scale), (T)(x.y * scale));
                if constexpr (DEF)
                    if (dfr) { const T f = deferred(n); v = mk<T>(f * v.x, f * v.y); }
                return v;
            });
        } else if (LEAN && !zrows && !deriv && !jo.hp && !(DEF && dfr)) {
            // no per-row factor: the flags stay off the element loop
            const C2<T>* src = reinterpret_cast<const C2<T>*>(stg);
            const T sc = (T)scale;
            regfft_load<T, N, DIR>(r, q, [&](int n) -> C2<T> {
                const C2<T> v = src[n * KT + c];
                return mk<T>(v.x * sc, v.y * sc);
            });
        } else if (LEAN && DIR > 0 && zrows && !deriv && !jo.hp && !(DEF && dfr)) {
            // the trimmed y inverse: masked rows read as zero (bit e: the e-th load)
            const C2<T>* src = reinterpret_cast<const C2<T>*>(stg);
            const T sc = (T)scale;
            int e = 0;   // load counter: a constant per call once the loads are unrolled
            regfft_load<T, N, DIR>(r, q, [&](int n) -> C2<T> {
                C2<T> v = src[n * KT + c];
                if (!((keepm >> e) & 1u)) v = mk<T>((T)0, (T)0);
                e++;
                return mk<T>(v.x * sc, v.y * sc);
            });
        } else {
            const C2<T>* src = reinterpret_cast<const C2<T>*>(stg);
            const T sc = (T)scale;
            regfft_load<T, N, DIR>(r, q, [&](int n) -> C2<T> {
                C2<T> v = src[n * KT + c];
                if (zrows && !keep[n]) v = mk<T>((T)0, (T)0);
                if constexpr (DEF)
                    if (dfr) { const T f = (T)deferred(n); v = mk<T>(f * v.x, f * v.y); }
                if (deriv) {
                    const T kk = deriv == 1 ? kax[n] + (T)kshift : (T)(deriv == 2 ? kout : kcol);
                    v = mk<T>(-kk * v.y, kk * v.x);
                }
                if (jo.hp) {
                    const double kn = a.axis == 0 ? a.g.kx[n] : a.g.ky[n];
                    if (!(kn * kn + kout * kout + kcol * kcol > a.hp_k2)) v = mk<T>((T)0, (T)0);
                }
                return mk<T>(v.x * sc, v.y * sc);
            });
        }
        __syncthreads();   // every thread has read the stage
        const int tn = t + NST * gridDim.x;
        if (tid == 0 && tn < total) {
            fence_proxy_async_smem();
            issue(tn, s);
        }
        const size_t base = a.axis == 0 ? (size_t)o * a.g.nzs : (size_t)o * a.g.ny * a.g.nzs;
        C2<T>* out = (C2<T>*)jo.out + (size_t)box * a.out_box_ch * a.g.ncs + base + k0;
        // outputs this thread stores: its column inside the box, and in a
        // row-filtered pass the kept rows (bit e: the e-th store of the last
        // stage)
        const bool col_ok = c < kt;
        const uint32_t smask = !col_ok ? 0u : (DIR < 0 && a.row_filter ? keepm : ~0u);
        if (skip) continue;
        int e = 0;   // store counter: a constant per call once the stores are unrolled
        regfft_run<T, N, DIR>(
            r, q, tw, [&](int L) { return xbuf + (size_t)L * KT + c; },
            [&](int k, C2<T> v) {
                if constexpr (LEAN) {
                    if ((smask >> e) & 1u) out[k * stride + c] = v;
                    e++;
                } else if (col_ok) {
                    out[k * stride + c] = v;
                }
            });
    }
    if (aborted) {
        if (tid == 0) {
            atomicExch(a.err, 2);
            for (int s = 0; s < NST; s++) mbar_wait(&bar[s], (uint32_t)(((i + s) / NST) & 1), SPK_WAIT_ITERS);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// z pass on the register FFT.  A CTA owns L consecutive (i,j) lines:
//  1. one bulk copy per input channel brings the L half spectra (rows of
//     nzs complex) into shared memory;
//  2. the input channels, paired into complex sequences Z = A + iB
//     (Hermitian-extended, DC/Nyquist imaginary parts dropped), are
//     inverse-transformed; the real fields go to shared memory;
//  3. one pass over the points forms the maxima of |u|, |B| for compute_dt
//     (compute_dt.cu:82-101,196-210), the real B lines for the anisotropic
//     STS flux, and the products -- TracelessShearMatrix[MHD]
//     (cuda_kernels.cu:39-55, 216-234), MagneticEmf (:240-252),
//     EnergyFluxVector (:277-289), ComputeBGradTheta +
//     ComputeAnisotropicHeatFlux (:360-383) -- as pairs (two real planes in
//     FP64, complex pairs in FP32) in the input area, which is free by then;
//  4. the product pairs are forward-transformed and unpacked into the half
//     spectra of each product (their D2Z), kz < kz_keep.
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared-memory carve of k_zpass2 (host and device agree through this):
// barrier, twiddle tables, input half spectra (later: the product pairs),
// real fields, exchange slots.
struct ZSmem { size_t tw, zero, junk, area, real, xb, cw, bre, total; };
// alias: the plain variant with one round of transforms in each direction
// and at least two FFT stages keeps its exchange slots in the input/product
// area: every slot has loaded its legs before the first exchange barrier (a
// one-stage transform has no such barrier before its stores to the slots)
__host__ __device__ inline bool zpass_alias(int gen, int nstages, int npin, int npout, int lines, int slots) {
    return gen == 0 && nstages >= 2 && npin * lines <= slots && npout * lines <= slots;
}
// Exchange slots of the z pass pad one element per 128-byte row of complex
// elements (16 in FP32, 8 in FP64), which keeps the exchanges of the
// register FFT free of bank conflicts in both precisions.
__host__ __device__ constexpr int zpass_xblock(int csz) { return 128 / csz; }
__host__ __device__ inline ZSmem zsmem_layout(int n, int twn, int csz, int nin, int nin_all, int npout, int lines,
                                              int nzs, int slots, int ncw, bool alias, int nbre = 0) {
    ZSmem z;
    const int rs = n + 16, xs = n + n / zpass_xblock(csz);
    z.tw = 128;
    z.zero = align16(z.tw + (size_t)twn * csz);              // a zero half spectrum (missing pair partner)
    z.junk = align16(z.zero + (size_t)nzs * csz);            // a real row that idle transforms write
    z.area = align16(z.junk + (size_t)rs * (csz / 2));
    const size_t raw = (size_t)nin * lines * nzs * csz, prod = (size_t)npout * lines * n * csz;
    const size_t xbs = (size_t)slots * xs * csz;
    size_t area = raw > prod ? raw : prod;
    if (alias && xbs > area) area = xbs;
    z.real = align16(z.area + area);
    const size_t realb = (size_t)nin_all * lines * rs * (csz / 2);
    // with aliased slots the block-max scratch (8 x 32 values) moves to the
    // real fields, which a few short lines per CTA do not cover
    const size_t redb = (size_t)8 * 32 * (csz / 2);
    z.xb = alias ? z.area : align16(z.real + realb);
    const size_t end = alias ? z.real + (realb > redb ? realb : redb) : z.xb + xbs;
    z.cw = align16(end);                                     // closure MLP parameters (floats)
    // the flux mode's real B lines (nbre components), bulk-copied with the inputs
    z.bre = align16(z.cw + (size_t)ncw * sizeof(float));
    z.total = align16(z.bre + (size_t)nbre * lines * n * (csz / 2));
    return z;
}

// The flux mode stages the CTA's lines of the cached real B in shared memory
// when a line's bytes keep every bulk copy 16-byte aligned.
template <typename T, int N> __host__ __device__ constexpr bool zpass_stage_b() { return (N * sizeof(T)) % 16 == 0; }

// GEN: 0 -- every input channel is a plain half spectrum; 1 -- derived
// gradient channels or the to-real output (the general path); 2 -- the
// general path with the learned closure (its own instantiation, so that the
// MLP's registers do not weigh on the others); 3 -- the same with the
// closure's tensor network (variant 3).
template <typename T, int N, int GEN>
__global__ void __launch_bounds__(128, GEN == 0 ? (sizeof(T) == 4 ? 6 : 5) : 4) k_zpass2(const __grid_constant__ ZArgs a) {
    using F = RegFft<T, N>;
    constexpr int LTPC = F::LTPC, TPC = F::TPC;
    constexpr int RS = N + 16;            // real rows: consecutive lines start 16 words apart in bank
    constexpr int XB = zpass_xblock((int)sizeof(C2<T>));
    constexpr int XS = N + N / XB;        // exchange slot (one pad element per XB)
    if (a.gate && a.gate_stage > a.gate->s_rkl) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int L = a.lines, nzs = a.g.nzs;
    const int nlines = a.g.nx * a.g.ny;
    // CTAs of box b cover lines [b*nlines, (b+1)*nlines); L divides nlines when nb > 1
    const int blocks_per_box = (nlines + L - 1) / L;
    const int box = blockIdx.x / blocks_per_box;
    const int line0 = (blockIdx.x - box * blocks_per_box) * L;
    const int nl = min(L, nlines - line0);
    const int nin = a.nin;
    const int nder0 = nin + (a.derive_gz == 1 ? 1 : 0);   // first closure d/dz channel
    const int nin_all = nder0 + (GEN >= 2 ? a.zder_n : 0);
    const int npin = (nin_all + 1) / 2, npout = (a.nout + 1) / 2;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int slots = nthr >> LTPC;
    const int sigma = tid >> LTPC, q = tid & (TPC - 1);
    const int sigma_w = (tid & ~31) >> LTPC;   // the lowest slot of this warp (warp-uniform)
    const bool clos = GEN >= 2 && a.closure;
    const bool alias = zpass_alias(GEN, F::NS, npin, npout, L, slots);
    // flux mode: the CTA's real B lines arrive with the inputs, off the point loop's path
    const bool stage_b = GEN == 1 && zpass_stage_b<T, N>() && a.load_breal;
    const ZSmem lay = zsmem_layout(N, F::TWN, (int)sizeof(C2<T>), nin, nin_all, npout, L, nzs, slots,
                                   clos ? (GEN == 3 ? C3_ZBYTES / 4 : CL_NP) : 0, alias, stage_b ? 3 : 0);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
    C2<T>* tw = reinterpret_cast<C2<T>*>(smem_raw + lay.tw);
    C2<T>* zrow = reinterpret_cast<C2<T>*>(smem_raw + lay.zero);
    T* junk = reinterpret_cast<T*>(smem_raw + lay.junk);
    C2<T>* raw = reinterpret_cast<C2<T>*>(smem_raw + lay.area);
    // the product pairs reuse the input area: pair p of line l takes the 2N
    // reals at (p*L + l)*2N.  FP64: two planes (channel 2p, then 2p+1), whose
    // 8-byte stores from the point loop are free of bank conflicts (the
    // plain pass is bound by shared-memory wavefronts).  FP32: interleaved
    // complex pairs, one load per leg of the forward transform (the FP32
    // pass is bound by instruction issue).
    constexpr bool PLANES = sizeof(T) == 8;
    constexpr int CS = PLANES ? N : 1;    // reals from channel 2p to 2p+1
    T* prodT = reinterpret_cast<T*>(raw);
    T* real = reinterpret_cast<T*>(smem_raw + lay.real);
    C2<T>* xb = reinterpret_cast<C2<T>*>(smem_raw + lay.xb);
    float* cw = reinterpret_cast<float*>(smem_raw + lay.cw);
    T* bre = reinterpret_cast<T*>(smem_raw + lay.bre);
    if (clos) {   // visible after the next barrier
        if constexpr (GEN == 3) {
            // the packed BF16 network, in 16-byte words
            const uint4* src = reinterpret_cast<const uint4*>(a.cparams);
            for (int i = tid; i < C3_FWD_BYTES / 16; i += nthr) reinterpret_cast<uint4*>(cw)[i] = src[i];
        } else {
            for (int i = tid; i < CL_NP; i += nthr) cw[i] = a.cparams[i];
        }
    }
    const C2<T>* in = (const C2<T>*)a.in + (size_t)box * a.in_box;
    DevScalars* bsc = a.scs + box;
    const int LRS = L * RS;

    // 1. one bulk copy per input channel: the CTA's lines are contiguous
    //    (rows of nzs elements, padding included: fewer, larger copies)
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = (uint32_t)((size_t)nl * nzs * sizeof(C2<T>));
        const uint32_t bbytes = stage_b ? (uint32_t)((size_t)nl * N * sizeof(T)) : 0u;
        mbar_expect_tx(bar, bytes * (uint32_t)nin + 3u * bbytes);
        for (int ch = 0; ch < nin; ch++)
            bulk_load(raw + (size_t)ch * L * nzs, in + (size_t)ch * a.cs_in + (size_t)line0 * nzs, bytes, bar);
        if (stage_b)
            for (int cb = 0; cb < 3; cb++)
                bulk_load(bre + (size_t)cb * L * N, (const T*)a.breal + ((size_t)cb * nlines + line0) * N, bbytes, bar);
    }
    regfft_fill_twiddles<T, N>(tw, (const C2<T>*)a.plan.tw, tid, nthr);
    for (int i = tid; i < nzs; i += nthr) zrow[i] = mk<T>((T)0, (T)0);
    const bool ok = mbar_wait(bar, 0, SPK_WAIT_ITERS);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            atomicExch(&bsc->err, 2);
            mbar_wait(bar, 0, SPK_WAIT_ITERS);   // bounded drain of the copies in flight
        }
        __syncthreads();
        return;
    }

    // no masked content: the inverse passes left kz >= kz_keep unwritten, and
    // those modes enter as zero
    const int kzk = (a.trim && !bsc->masked_live) ? a.g.kz_keep : nzs;
    auto xaddr = [&](int Lx) { return xb + (size_t)sigma * XS + padb<XB>(Lx); };
    C2<T> r[F::E];

    // 2. inverse transforms of the input pairs
    const int ninv = npin * L;
    for (int base = 0; base < ninv; base += slots) {
        const int tau = base + sigma;
        const bool valid = tau < ninv;
        const int p = valid ? tau / L : 0, l = valid ? tau - p * L : 0;
        // false: no slot of this warp has a transform, and the warp skips the math
        const bool act = base + sigma_w < ninv;
        const C2<T>* pa = raw + (size_t)(2 * p * L + l) * nzs;
        const C2<T>* pb = 2 * p + 1 < nin ? pa + (size_t)L * nzs : zrow;
        auto chv = [&](int ch, int k) -> C2<T> {
            if (k >= kzk) return mk<T>((T)0, (T)0);
            if (ch < nin) {
                C2<T> v = raw[((size_t)ch * L + l) * nzs + k];
                if (a.derive_gz == 2 && ch == a.ch_th) {
                    const T kz = (T)a.g.kz[k];
                    v = mk<T>(-kz * v.y, kz * v.x);
                }
                return v;
            }
            if (ch == nin && a.derive_gz == 1) {
                const C2<T> th = raw[((size_t)a.ch_th * L + l) * nzs + k];
                const T kz = (T)a.g.kz[k];
                return mk<T>(-kz * th.y, kz * th.x);
            }
            if (ch >= nder0 && ch < nin_all) {   // closure: d/dz of u [and B]
                const C2<T> x = raw[((size_t)a.zder_src[ch - nder0] * L + l) * nzs + k];
                const T kz = (T)a.g.kz[k];
                return mk<T>(-kz * x.y, kz * x.x);
            }
            return mk<T>((T)0, (T)0);
        };
        if (act) regfft_load<T, N, +1>(r, q, [&](int n) -> C2<T> {
            constexpr int NH = N >> 1;
            const int k = n <= NH ? n : N - n;
            C2<T> A, B;
            if constexpr (GEN == 0) {
                const C2<T> zz = mk<T>((T)0, (T)0);
                A = k < kzk ? pa[k] : zz;
                B = k < kzk ? pb[k] : zz;
            } else {
                A = chv(2 * p, k);
                B = chv(2 * p + 1, k);
            }
            if (n == 0 || n == NH) return mk<T>(A.x, B.x);
            if (n < NH) return mk<T>(A.x - B.y, A.y + B.x);
            return mk<T>(A.x + B.y, B.x - A.y);
        });
        // an idle transform (and the missing partner of an odd last pair) writes the junk row
        T* pr0 = valid ? real + (size_t)(2 * p * L + l) * RS : junk;
        T* pr1 = (valid && 2 * p + 1 < nin_all) ? pr0 + LRS : junk;
        const bool to_real = GEN != 0 && a.mode == ZM_TO_REAL && valid && l < nl;
        regfft_run<T, N, +1, false, XB>(r, q, tw, xaddr, [&](int z, C2<T> v) {
            pr0[z] = v.x;
            pr1[z] = v.y;
            if (GEN != 0 && to_real) {
                const size_t line = (size_t)(line0 + l);
                if (2 * p < nin) a.real_out[((size_t)(2 * p) * nlines + line) * N + z] = (double)v.x;
                if (2 * p + 1 < nin) a.real_out[((size_t)(2 * p + 1) * nlines + line) * N + z] = (double)v.y;
            }
        }, act);
    }
    __syncthreads();
    if (a.mode == ZM_TO_REAL) return;

    // 3. one pass over the points: CFL maxima, real B for the STS flux, and
    //    the products, stored as complex pairs (channel 2p, 2p+1)
    T* breal = (T*)a.breal;
    const bool want_prod = a.nout > 0;
    {
        T mu[8] = {(T)0, (T)0, (T)0, (T)0, (T)0, (T)0, (T)0, (T)0};
        int bad = 0;
        const T third = (T)(1.0 / 3.0);
        const size_t pstride = (size_t)L * N * 2;   // scalars between product pairs
        // the closure's gradient components of the point at fr (variant 2: all nine
        // of each field from ch_dx; else d/dx, d/dy and the z-derivative channels)
        auto grads = [&](const T* fr, float* A, float* G) {
            if (a.cl_grad9) {
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        A[3 * i + j] = (float)fr[(a.ch_dx + 3 * j + i) * LRS];
                        G[3 * i + j] = a.mhd ? (float)fr[(a.ch_dx + 9 + 3 * j + i) * LRS] : 0.f;
                    }
            } else {
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    A[3 * i + 0] = (float)fr[(a.ch_dx + i) * LRS];
                    A[3 * i + 1] = (float)fr[(a.ch_dy + i) * LRS];
                    A[3 * i + 2] = (float)fr[(nder0 + i) * LRS];
                    G[3 * i + 0] = a.mhd ? (float)fr[(a.ch_dx + 3 + i) * LRS] : 0.f;
                    G[3 * i + 1] = a.mhd ? (float)fr[(a.ch_dy + 3 + i) * LRS] : 0.f;
                    G[3 * i + 2] = a.mhd ? (float)fr[(nder0 + 3 + i) * LRS] : 0.f;
                }
            }
        };
        // variant 3 runs its network on the tensor cores per chunk of 128
        // points, ahead of the chunk's products; the others take all points
        // in one chunk
        unsigned char* c3rows = reinterpret_cast<unsigned char*>(cw) + C3_FWD_BYTES;
        const int EPC = GEN == 3 ? C3_ZCHUNK : L * N;
        // The products of incompressible HD and MHD alone (the RK3 step):
        // the general loop's arithmetic, in the same order, with its
        // per-point flag tests hoisted (one loop per field set).
        const bool hdmhd = GEN == 0 && want_prod && a.mode == ZM_PRODUCTS && a.hydro && !a.bous && !a.aniso &&
                           !a.load_breal && !a.store_breal && a.ch_u >= 0 && (!a.mhd || a.ch_b >= 0);
        auto hdmhd_loop = [&](auto mhd_c) {
            constexpr bool MHD = decltype(mhd_c)::value;
            const int cu = a.ch_u * LRS, cb = MHD ? a.ch_b * LRS : 0;
            const bool dmax = a.do_max != 0, odd = (a.nout & 1) != 0;
            for (int e = tid; e < L * N; e += nthr) {
                const int l = (int)((unsigned)e / (unsigned)N), z = e - l * N;
                const T* fr = real + (size_t)l * RS + z;
                const T ux = fr[cu], uy = fr[cu + LRS], uz = fr[cu + 2 * LRS];
                T bx = 0, by = 0, bz = 0;
                if constexpr (MHD) { bx = fr[cb]; by = fr[cb + LRS]; bz = fr[cb + 2 * LRS]; }
                if (dmax && l < nl) {
                    const T av[6] = {fabs(ux), fabs(uy), fabs(uz), fabs(bx), fabs(by), fabs(bz)};
#pragma unroll
                    for (int c = 0; c < 6; c++) {
                        if (!isfinite(av[c])) bad = 1;
                        mu[c] = fmax(mu[c], av[c]);
                    }
                }
                T* pp = prodT + (PLANES ? (size_t)l * 2 * N + z : ((size_t)l * N + z) * 2);
                auto put = [&](int ch, T v) { pp[(size_t)(ch >> 1) * pstride + (ch & 1) * CS] = v; };
                if constexpr (!MHD) {
                    put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz) * third);
                    put(1, ux * uy);
                    put(2, ux * uz);
                    put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz) * third);
                    put(4, uy * uz);
                } else {
                    put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz - (T)2.0 * bx * bx + by * by + bz * bz) * third);
                    put(1, ux * uy - bx * by);
                    put(2, ux * uz - bx * bz);
                    put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz + bx * bx - (T)2.0 * by * by + bz * bz) * third);
                    put(4, uy * uz - by * bz);
                    put(5, -by * uz + bz * uy + (T)0.f);
                    put(6, bx * uz - bz * ux + (T)0.f);
                    put(7, -bx * uy + by * ux + (T)0.f);
                }
                if (odd) put(a.nout, (T)0);
            }
        };
        // The anisotropic heat flux of an RKL2 stage (ZM_RKL_FLUX with the real
        // B lines staged): the general loop's arithmetic, in the same order,
        // with its per-point flag tests hoisted.
        const bool flux = GEN == 1 && stage_b && want_prod && a.mode == ZM_RKL_FLUX && a.aniso && !a.store_breal &&
                          !a.do_max && a.ch_u < 0 && a.derive_gz == 2 && a.ch_gx >= 0 && a.ch_gy >= 0 &&
                          a.shear_part == 0 && !clos;
        if (hdmhd) {
            if (a.mhd) hdmhd_loop(std::integral_constant<bool, true>());
            else hdmhd_loop(std::integral_constant<bool, false>());
        } else if (flux) {
            const int cgx = a.ch_gx * LRS, cgy = a.ch_gy * LRS, cgz = a.ch_th * LRS;
            const int sd = a.sd;
            const bool odd = (a.nout & 1) != 0;
            const T chi = (T)a.chi, W = (T)a.omegaT2;
            for (int e = tid; e < L * N; e += nthr) {
                const int l = (int)((unsigned)e / (unsigned)N), z = e - l * N;
                const T* fr = real + (size_t)l * RS + z;
                T bx = 0, by = 0, bz = 0;
                if (l < nl) {
                    bx = bre[(size_t)(0 * L + l) * N + z];
                    by = bre[(size_t)(1 * L + l) * N + z];
                    bz = bre[(size_t)(2 * L + l) * N + z];
                }
                const T gx = fr[cgx], gy = fr[cgy], gz = fr[cgz];
                T* pp = prodT + (PLANES ? (size_t)l * 2 * N + z : ((size_t)l * N + z) * 2);
                auto put = [&](int ch, T v) { pp[(size_t)(ch >> 1) * pstride + (ch & 1) * CS] = v; };
                const T bgt = bx * gx + by * gy + bz * gz;
                const T b2 = bx * bx + by * by + bz * bz;
                const T bs = sd == 0 ? bx : (sd == 1 ? by : bz);
                put(0, chi * bx * (bgt + W * bs) / b2);
                put(1, chi * by * (bgt + W * bs) / b2);
                put(2, chi * bz * (bgt + W * bs) / b2);
                if (odd) put(a.nout, (T)0);
            }
        } else
        for (int e0 = 0; e0 < L * N; e0 += EPC) {
        if constexpr (GEN == 3) {
            if (clos) {
                const int e = e0 + tid;
                float A[9], G[9];
                if (e < L * N) {
                    const int l = (int)((unsigned)e / (unsigned)N), z = e - l * N;
                    grads(real + (size_t)l * RS + z, A, G);
                } else {
#pragma unroll
                    for (int i = 0; i < 9; i++) A[i] = G[i] = 0.f;
                }
                c3_put_inputs(c3rows, tid, A, G);
                __syncthreads();
                c3_chunk_mlp(reinterpret_cast<const unsigned char*>(cw), c3rows, tid >> 5, tid & 31);
                __syncthreads();
            }
        }
        for (int e = e0 + tid; e < min(e0 + EPC, L * N); e += nthr) {
            const int l = (int)((unsigned)e / (unsigned)N), z = e - l * N;
            const bool live = l < nl;
            const size_t line = (size_t)(line0 + l);
            const T* fr = real + (size_t)l * RS + z;
            T ux = 0, uy = 0, uz = 0, bx = 0, by = 0, bz = 0, th = 0, gx = 0, gy = 0, gz = 0;
            if (a.ch_u >= 0) { ux = fr[a.ch_u * LRS]; uy = fr[(a.ch_u + 1) * LRS]; uz = fr[(a.ch_u + 2) * LRS]; }
            if (a.load_breal) {
                if (live && stage_b) {
                    bx = bre[(size_t)(0 * L + l) * N + z];
                    by = bre[(size_t)(1 * L + l) * N + z];
                    bz = bre[(size_t)(2 * L + l) * N + z];
                } else if (live) {
                    bx = breal[(0 * (size_t)nlines + line) * N + z];
                    by = breal[(1 * (size_t)nlines + line) * N + z];
                    bz = breal[(2 * (size_t)nlines + line) * N + z];
                }
            } else if (a.ch_b >= 0) {
                bx = fr[a.ch_b * LRS]; by = fr[(a.ch_b + 1) * LRS]; bz = fr[(a.ch_b + 2) * LRS];
            }
            if (live && a.store_breal) {
                breal[(0 * (size_t)nlines + line) * N + z] = bx;
                breal[(1 * (size_t)nlines + line) * N + z] = by;
                breal[(2 * (size_t)nlines + line) * N + z] = bz;
            }
            if (live && a.do_max) {
                const T av[6] = {fabs(ux), fabs(uy), fabs(uz), fabs(bx), fabs(by), fabs(bz)};
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    if (!isfinite(av[c])) bad = 1;
                    mu[c] = fmax(mu[c], av[c]);
                }
            }
            if (!want_prod) continue;
            if (a.ch_th >= 0 && a.derive_gz != 2) th = fr[a.ch_th * LRS];
            if (a.ch_gx >= 0) gx = fr[a.ch_gx * LRS];
            if (a.ch_gy >= 0) gy = fr[a.ch_gy * LRS];
            if (a.derive_gz == 1) gz = fr[nin * LRS];
            else if (a.derive_gz == 2) gz = fr[a.ch_th * LRS];
            T* pp = prodT + (PLANES ? (size_t)l * 2 * N + z : ((size_t)l * N + z) * 2);
            auto put = [&](int ch, T v) { pp[(size_t)(ch >> 1) * pstride + (ch & 1) * CS] = v; };
            int qc = 0;
            // learned closure: -2 nu_t S into the stress, -eta_t J into the EMF
            float ctau[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, cemf[3] = {0.f, 0.f, 0.f};
            if (clos) {
                float A[9], G[9], vn, ve;
                grads(fr, A, G);
                if constexpr (GEN == 3) {
                    // the network's outputs for this point, left in its row by the chunk pass
                    float f[8], S5[5], J3[3];
                    const float n = closure_features<float>(A, G, f, S5, J3);
                    const float* o12 = reinterpret_cast<const float*>(c3rows + (size_t)(e - e0) * C3_ZROW);
                    c3_terms(o12, a.delta2, n, A[8], S5, J3, a.mhd != 0, ctau, cemf, &vn, &ve);
                } else {
                    closure_point(cw, a.delta2, A, G, ctau, cemf, &vn, &ve);
                }
                if (live && a.do_max) {
                    if (!isfinite(vn) || !isfinite(ve)) bad = 1;
                    mu[6] = fmax(mu[6], (T)vn);
                    mu[7] = fmax(mu[7], (T)(a.mhd ? ve : 0.f));
                }
            }
            if constexpr (GEN == 1) {
                // ShearMatrix (cuda_kernels.cu:59-77) of the transfer spectra
                if (a.shear_part == 1) { put(0, ux * ux); put(1, ux * uy); put(2, ux * uz); qc = 3; }
                if (a.shear_part == 2) { put(0, uy * uy); put(1, uy * uz); put(2, uz * uz); qc = 3; }
            }
            if (a.mode == ZM_PRODUCTS) {
                if (a.hydro) {
                    if (!a.mhd) {
                        put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz) * third);
                        put(1, ux * uy);
                        put(2, ux * uz);
                        put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz) * third);
                        put(4, uy * uz);
                    } else {
                        put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz - (T)2.0 * bx * bx + by * by + bz * bz) * third);
                        put(1, ux * uy - bx * by);
                        put(2, ux * uz - bx * bz);
                        put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz + bx * bx - (T)2.0 * by * by + bz * bz) * third);
                        put(4, uy * uz - by * bz);
                    }
                    if (clos)
#pragma unroll
                        for (int r = 0; r < 5; r++) pp[(size_t)(r >> 1) * pstride + (r & 1) * CS] += (T)ctau[r];
                    qc = 5;
                }
                if (a.mhd) {
                    put(qc, -by * uz + bz * uy + (T)cemf[0]);
                    put(qc + 1, bx * uz - bz * ux + (T)cemf[1]);
                    put(qc + 2, -bx * uy + by * ux + (T)cemf[2]);
                    qc += 3;
                }
                if (a.bous) {
                    put(qc, ux * th); put(qc + 1, uy * th); put(qc + 2, uz * th);
                    qc += 3;
                }
            }
            if (a.aniso) {
                const T bgt = bx * gx + by * gy + bz * gz;
                const T b2 = bx * bx + by * by + bz * bz;
                const T bs = a.sd == 0 ? bx : (a.sd == 1 ? by : bz);
                const T chi = (T)a.chi, W = (T)a.omegaT2;
                put(qc, chi * bx * (bgt + W * bs) / b2);
                put(qc + 1, chi * by * (bgt + W * bs) / b2);
                put(qc + 2, chi * bz * (bgt + W * bs) / b2);
                qc += 3;
            }
            if (a.nout & 1) put(a.nout, (T)0);
        }
        if constexpr (GEN == 3) {
            if (clos) __syncthreads();   // the chunk's outputs are read before the next chunk's inputs
        }
        }
        if (a.do_max) {
            // block-max scratch (8 x 32): the exchange slots, or with aliased
            // slots the real fields (every warp has left the point loop)
            T* red = reinterpret_cast<T*>(xb);
            if (alias) {
                __syncthreads();
                red = real;
            }
            const int nmax = clos ? 8 : 6;
            warp_block_max<T>(mu, nmax, red);
            if (tid < nmax) {
                const double m = (double)red[tid * 32];
                const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
                unsigned long long* dst = bsc->maxbits + tid;
                if (bits > *((volatile unsigned long long*)dst)) atomicMax(dst, bits);
            }
            if (bad) atomicOr(&bsc->nonfinite, 1);
        }
    }
    if (!want_prod) return;
    __syncthreads();   // products written; the block-max scratch read

    // 4. forward transforms of the product pairs, unpacked half spectra
    const int kk = a.g.kz_keep;
    C2<T>* out = (C2<T>*)a.out + (size_t)box * a.out_box;
    const T half = (T)0.5;
    const int lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;
    const int nfw = npout * L;
    for (int base = 0; base < nfw; base += slots) {
        if (base > 0) __syncthreads();   // the previous round's unpack has read the exchange slots
        const int tau = base + sigma;
        const bool valid = tau < nfw;
        const int p = valid ? tau / L : 0, l = valid ? tau - p * L : 0;
        const T* pp = prodT + (size_t)(p * L + l) * 2 * N;
        // (forward rounds: FP64 only; in FP32 the branches cost more than they save, measured)
        const bool act = sizeof(T) == 4 || base + sigma_w < nfw;
        if (act) regfft_load<T, N, -1>(r, q, [&](int z) -> C2<T> {
            if constexpr (PLANES) return mk<T>(pp[z], pp[N + z]);
            else return reinterpret_cast<const C2<T>*>(pp)[z];
        });
        regfft_run<T, N, -1, true, XB>(r, q, tw, xaddr, [&](int k, C2<T> v) { *xaddr(k) = v; }, act);
        __syncthreads();
        for (int s2 = warp; s2 < slots; s2 += nwarp) {
            const int tau2 = base + s2;
            if (tau2 >= nfw) break;
            const int p2 = tau2 / L, l2 = tau2 - p2 * L;
            if (l2 >= nl) continue;
            const C2<T>* Z = xb + (size_t)s2 * XS;
            const size_t off0 = (size_t)(line0 + l2) * nzs;
            C2<T>* o0 = out + (size_t)(2 * p2) * a.cs_out + off0;
            C2<T>* o1 = out + (size_t)(2 * p2 + 1) * a.cs_out + off0;
            const bool two = 2 * p2 + 1 < a.nout;
            for (int k = lane; k < kk; k += 32) {
                const C2<T> zk = Z[padb<XB>(k)], zm = Z[padb<XB>(k ? N - k : 0)];
                o0[k] = mk<T>(half * (zk.x + zm.x), half * (zk.y - zm.y));
                if (two) o1[k] = mk<T>(half * (zk.y + zm.y), half * (zm.x - zk.x));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// RHS, Leray projection and time update, one mode per thread, after the
// x-forward pass has transformed the products:
//   NonLinHydroAdv (cuda_kernels.cu:82-98), MagneticShear (:257-272),
//   NonLinBoussinesqAdv (:293-304) with the 2/3 mask (DivergenceMask,
//   cuda_kernels_generic.cu:315-334), BoussinesqStrat (:310-325), the
//   parabolic terms (physics.cu:145-230: nablaOpVector/Scalar, or the
//   anisotropic flux divergence of AnisotropicHeatFlux), GradPseudoPressure
//   (:128-159), and axpyComplex of RungeKutta3 / ForwardEuler
//   (hydro_mhd_advance.cu:79-248), with CleanDivergence of the next step
//   (cuda_kernels_generic.cu:288-313) on the last stage.
// ---------------------------------------------------------------------------
// New state value of one mode given its RK scratch value S (read up front).
__device__ __forceinline__ double2 rk_value(const XfArgs& a, size_t gi, double2 X, double2 S, double2 R, double dt) {
    const double g0 = 8.0 / 15.0, g1 = 5.0 / 12.0, g2 = 3.0 / 4.0, x0 = -17.0 / 60.0, x1 = -5.0 / 12.0;
    switch (a.mode) {
        case XM_RK0: {
            // U1 = U + g0 dt R, then S = U1 + x0 dt R (the second axpyComplex
            // reads the already-updated fields, hydro_mhd_advance.cu:119-122)
            const double bu = g0 * dt, bs = x0 * dt;
            const double2 Un = d2(1.0 * X.x + bu * R.x, 1.0 * X.y + bu * R.y);
            a.S[gi] = d2(1.0 * Un.x + bs * R.x, 1.0 * Un.y + bs * R.y);
            return Un;
        }
        case XM_RK1: {
            const double bu = g1 * dt, bs = x1 * dt;
            const double2 Un = d2(1.0 * S.x + bu * R.x, 1.0 * S.y + bu * R.y);
            a.S[gi] = d2(1.0 * Un.x + bs * R.x, 1.0 * Un.y + bs * R.y);
            return Un;
        }
        case XM_RK2: {
            const double bu = g2 * dt;
            return d2(1.0 * S.x + bu * R.x, 1.0 * S.y + bu * R.y);
        }
        case XM_EULER:
            return d2(1.0 * X.x + dt * R.x, 1.0 * X.y + dt * R.y);
        default:
            a.out[gi] = R;
            return X;
    }
}

// MINB: resident CTAs per SM the registers are budgeted for (4 for the FP32
// HD/MHD form, where the few spills cost less than the lost occupancy; 3 for
// the FP64 form and for Boussinesq, which keep more values live).
template <typename T, int MINB>
__global__ void __launch_bounds__(128, MINB) k_rhs(const __grid_constant__ XfArgs a, FastDiv fzh) {
    const size_t nc = a.g.nc;
    const int nzh = a.g.nzh, nzs = a.g.nzs;
    const unsigned ny = (unsigned)a.g.ny, nlines = (unsigned)(a.g.nx * a.g.ny);
    const bool needS = a.mode == XM_RK1 || a.mode == XM_RK2;
    const double2 z0 = d2(0.0, 0.0);
    // deferred masked modes: every stage visits the kept modes only
    // (k_masked_rk moves the masked ones once per step)
    const bool compact = a.defer != 0;
    const int kzk = a.g.kz_keep;
    const size_t total = (compact ? (size_t)a.nkx * a.nky * kzk : nc) * (size_t)a.nb;
    const double shx = grid_shx(a.g);   // shearing box: kx = kx0 + shx ky
    // One copy of the mode loop with the flags of incompressible MHD (no
    // Boussinesq, stratification, shearing box or super-time-stepping) fixed
    // at compile time, which keeps the unused fields' registers out of it;
    // the general copy serves every other configuration.  Same arithmetic.
    auto modes = [&](auto mhd_only) {
        constexpr bool ONLY = decltype(mhd_only)::value;
        const bool INC = ONLY || a.incompressible, MHD = ONLY || a.mhd, BOUS = !ONLY && a.bous;
        const bool STRAT = !ONLY && a.strat, SHEAR = !ONLY && a.g.shear != 0.0;
        const unsigned stsm = ONLY ? 0u : a.sts_mask;
        for (size_t gb = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gb < total; gb += (size_t)gridDim.x * blockDim.x) {
            int k, i, j, box;
            unsigned line;
            if (compact) {
                // compact index -> box, kept x index, kept y index, k < kz_keep
                const unsigned r1 = a.fd_kzk.div((unsigned)gb);
                k = (int)(gb - (size_t)r1 * kzk);
                const unsigned r2 = a.fd_nky.div(r1);
                const int jy = (int)(r1 - r2 * (unsigned)a.nky);
                const unsigned r3 = a.fd_nkx.div(r2);
                const int ix = (int)(r2 - r3 * (unsigned)a.nkx);
                box = (int)r3;
                i = a.kxi[ix];
                j = a.kyi[jy];
                line = (unsigned)i * ny + (unsigned)j;
            } else {
                // global line over the boxes -> box, line, k (nx*ny is a power of two)
                const unsigned gline = fzh.div((unsigned)gb);
                k = (int)(gb - (size_t)gline * nzh);
                const unsigned ubox = a.fd_nl.div(gline);
                box = (int)ubox;
                line = gline - ubox * nlines;
                const unsigned ui = a.fd_ny.div(line);
                i = (int)ui;
                j = (int)(line - ui * ny);
            }
            const size_t gi = (size_t)line * nzh + k;                // mode within the box
            const size_t bo = (size_t)box * a.box_state;            // box offset in U, S, out
            const double dt = a.sc[box].dt, nu = a.sc[box].nu, nu_m = a.sc[box].nu_m, nu_th = a.sc[box].nu_th;
            // compact: every visited mode is kept (kxi and kyi list the indices of
            // nonzero mask factors, and the kz mask is the prefix k < kz_keep), so
            // the product loads need not wait for the mask tables
            const bool m = compact || (a.g.mx[i] != 0.0 && a.g.my[j] != 0.0 && a.g.mz[k] != 0.0);

            const C2<T>* nl = (const C2<T>*)a.nl + (size_t)box * a.box_nl;
            const size_t li = (size_t)line * nzs + k;   // products: [ch][line][nzs]
            auto P = [&](int ch) -> double2 { return to_d2(nl[(size_t)ch * a.cs_nl + li]); };

            // every load of the mode first (state, RK scratch, products), so that
            // they are all in flight together
            double2 Xu[3] = {z0, z0, z0}, Xb[3] = {z0, z0, z0}, Xt = z0;
            double2 Su[3] = {z0, z0, z0}, Sb[3] = {z0, z0, z0}, St = z0;
            double2 t0 = z0, t1 = z0, t2 = z0, t3 = z0, t4 = z0, e0 = z0, e1 = z0, e2 = z0;
            double2 f0 = z0, f1 = z0, f2 = z0, q0 = z0, q1 = z0, q2 = z0;
            if (INC) {
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    Xu[c] = a.U[bo + (size_t)(a.VEL + c) * nc + gi];
                    if (needS) Su[c] = a.S[bo + (size_t)(a.VEL + c) * nc + gi];
                }
            }
            if (MHD) {
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    Xb[c] = a.U[bo + (size_t)(a.MAG + c) * nc + gi];
                    if (needS) Sb[c] = a.S[bo + (size_t)(a.MAG + c) * nc + gi];
                }
            }
            if (BOUS) {
                Xt = a.U[bo + (size_t)a.TH * nc + gi];
                if (needS) St = a.S[bo + (size_t)a.TH * nc + gi];
            }
            if (m) {
                if (INC && a.nl_T >= 0) { t0 = P(a.nl_T); t1 = P(a.nl_T + 1); t2 = P(a.nl_T + 2); t3 = P(a.nl_T + 3); t4 = P(a.nl_T + 4); }
                if (MHD && a.nl_E >= 0) { e0 = P(a.nl_E); e1 = P(a.nl_E + 1); e2 = P(a.nl_E + 2); }
                if (BOUS && a.nl_F >= 0) { f0 = P(a.nl_F); f1 = P(a.nl_F + 1); f2 = P(a.nl_F + 2); }
                if (BOUS && a.aniso_rhs && a.nl_Q >= 0) { q0 = P(a.nl_Q); q1 = P(a.nl_Q + 1); q2 = P(a.nl_Q + 2); }
            }
            const double kx = a.g.kx[i] + shx * a.g.ky[j], ky = a.g.ky[j], kz = a.g.kz[k];
            const double k2 = kx * kx + ky * ky + kz * kz;
            double2 usd = z0;

            if (INC) {
                double2 R[3];
                // -i * mask * k_j T_ij with T = [[t0 t1 t2] [t1 t3 t4] [t2 t4 -t0-t3]]
                const double2 s0 = d2(kx * t0.x + ky * t1.x + kz * t2.x, kx * t0.y + ky * t1.y + kz * t2.y);
                const double2 s1 = d2(kx * t1.x + ky * t3.x + kz * t4.x, kx * t1.y + ky * t3.y + kz * t4.y);
                const double2 s2 = d2(kx * t2.x + ky * t4.x - kz * (t0.x + t3.x), kx * t2.y + ky * t4.y - kz * (t0.y + t3.y));
                R[0] = d2(s0.y, -s0.x);
                R[1] = d2(s1.y, -s1.x);
                R[2] = d2(s2.y, -s2.x);
                if (STRAT) {
                    if (a.sd == 0)      { R[0] = d2(R[0].x - Xt.x, R[0].y - Xt.y); usd = Xu[0]; }
                    else if (a.sd == 1) { R[1] = d2(R[1].x - Xt.x, R[1].y - Xt.y); usd = Xu[1]; }
                    else                { R[2] = d2(R[2].x - Xt.x, R[2].y - Xt.y); usd = Xu[2]; }
                }
                if (SHEAR) {
                    // BackgroundShear / BackgroundRotation (shear_rotation.cu:11-63):
                    // dvy += S vx; with rotation dvx += 2 omega vy, dvy -= 2 omega vx
                    const double S = a.g.shear;
                    R[1] = d2(R[1].x + S * Xu[0].x, R[1].y + S * Xu[0].y);
                    if (a.rotating) {
                        const double w2 = 2.0 * a.omega;
                        R[0] = d2(R[0].x + w2 * Xu[1].x, R[0].y + w2 * Xu[1].y);
                        R[1] = d2(R[1].x - w2 * Xu[0].x, R[1].y - w2 * Xu[0].y);
                    }
                }
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    if (!((stsm >> (a.VEL + c)) & 1u)) {
                        const double f = -nu * k2;
                        R[c] = d2(R[c].x + f * Xu[c].x, R[c].y + f * Xu[c].y);
                    }
                }
                // Leray: dU += i k (i k.dU)/k^2; the shearing box adds S ky vx to
                // k.dU (GradPseudoPressureShearing, cuda_kernels.cu:165-196)
                const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
                double sx, sy;
                if (SHEAR) {
                    const double Sky = a.g.shear * ky;
                    sx = Sky * Xu[0].x + kx * R[0].x + ky * R[1].x + kz * R[2].x;
                    sy = Sky * Xu[0].y + kx * R[0].y + ky * R[1].y + kz * R[2].y;
                } else {
                    sx = kx * R[0].x + ky * R[1].x + kz * R[2].x;
                    sy = kx * R[0].y + ky * R[1].y + kz * R[2].y;
                }
                const double kk[3] = {kx, ky, kz};
    #pragma unroll
                for (int c = 0; c < 3; c++) R[c] = d2(R[c].x - kk[c] * ik2 * sx, R[c].y - kk[c] * ik2 * sy);
                double2 Un[3];
    #pragma unroll
                for (int c = 0; c < 3; c++) Un[c] = rk_value(a, bo + (size_t)(a.VEL + c) * nc + gi, Xu[c], Su[c], R[c], dt);
                if (a.mode != XM_DFIELD) {
                    if (a.clean) clean3(Un, kx, ky, kz);
    #pragma unroll
                    for (int c = 0; c < 3; c++) a.U[bo + (size_t)(a.VEL + c) * nc + gi] = Un[c];
                }
            }

            if (MHD) {
                // i * mask * (k x E)
                const double2 S3[3] = {d2(ky * e2.x - kz * e1.x, ky * e2.y - kz * e1.y),
                                       d2(kz * e0.x - kx * e2.x, kz * e0.y - kx * e2.y),
                                       d2(kx * e1.x - ky * e0.x, kx * e1.y - ky * e0.y)};
                double2 Un[3];
    #pragma unroll
                for (int c = 0; c < 3; c++) {
                    double2 R = d2(-S3[c].y, S3[c].x);
                    // shearing box: dBy -= S Bx (ShearingFlow with -shear)
                    if (c == 1 && SHEAR) R = d2(R.x + (-a.g.shear) * Xb[0].x, R.y + (-a.g.shear) * Xb[0].y);
                    if (!((stsm >> (a.MAG + c)) & 1u)) {
                        const double f = -nu_m * k2;
                        R = d2(R.x + f * Xb[c].x, R.y + f * Xb[c].y);
                    }
                    Un[c] = rk_value(a, bo + (size_t)(a.MAG + c) * nc + gi, Xb[c], Sb[c], R, dt);
                }
                if (a.mode != XM_DFIELD) {
                    if (a.clean) clean3(Un, kx, ky, kz);
    #pragma unroll
                    for (int c = 0; c < 3; c++) a.U[bo + (size_t)(a.MAG + c) * nc + gi] = Un[c];
                }
            }

            if (BOUS) {
                const double2 s = d2(kx * f0.x + ky * f1.x + kz * f2.x, kx * f0.y + ky * f1.y + kz * f2.y);
                double2 R = d2(s.y, -s.x);   // -i * mask * k.(u theta)
                if (STRAT) R = d2(R.x + a.N2 * usd.x, R.y + a.N2 * usd.y);
                if (!((stsm >> a.TH) & 1u)) {
                    if (a.aniso_rhs) {
                        const double2 sq = d2(kx * q0.x + ky * q1.x + kz * q2.x, kx * q0.y + ky * q1.y + kz * q2.y);
                        R = d2(R.x - sq.y, R.y + sq.x);   // += i * mask * k.q
                    } else {
                        const double f = -nu_th * k2;
                        R = d2(R.x + f * Xt.x, R.y + f * Xt.y);
                    }
                }
                const double2 Un = rk_value(a, bo + (size_t)a.TH * nc + gi, Xt, St, R, dt);
                if (a.mode != XM_DFIELD) a.U[bo + (size_t)a.TH * nc + gi] = Un;
            }
        }
    };
    if (a.incompressible && a.mhd && !a.bous && !a.strat && a.g.shear == 0.0 && a.sts_mask == 0)
        modes(std::integral_constant<bool, true>());
    else
        modes(std::integral_constant<bool, false>());
}

// ---------------------------------------------------------------------------
// RKL2 stage of the anisotropic heat flux, one mode per thread, after the
// x-forward pass has transformed the three flux components:
// dtheta = i * mask * k.q (AnisotropicHeatFlux divergence,
// anisotropic_conduction.cu:10-62) and the RKL2 stage update of
// compute_cycle_RKL2 (rkl.cu:437-591).  Skipped for stages beyond the
// cycle's stage count.
// ---------------------------------------------------------------------------
// Masked modes of a deferred RK3 step, once per step (with stage 2):
// outside the 2/3 mask the right-hand side is the diffusion -nu k^2 U of a
// divergence-free U (the nonlinear terms are masked and the Leray
// projection leaves it unchanged), so the three stages amount to
// U <- c(z) U, z = -nu k^2 dt, c from the recurrences of rk_value; the
// divergence cleaning of the next step follows, as in k_rhs.  Kept modes are
// skipped (k_rhs owns them).
__global__ void __launch_bounds__(256) k_masked_rk(const __grid_constant__ XfArgs a, FastDiv fzh) {
    const size_t nc = a.g.nc;
    const int nzh = a.g.nzh;
    const unsigned ny = (unsigned)a.g.ny, nlines = (unsigned)(a.g.nx * a.g.ny);
    const size_t total = nc * (size_t)a.nb;
    const double g0 = 8.0 / 15.0, g1 = 5.0 / 12.0, g2 = 3.0 / 4.0, x0 = -17.0 / 60.0, x1 = -5.0 / 12.0;
    auto amp = [&](double z) {
        const double c1 = 1.0 + g0 * z;
        const double s1 = c1 + x0 * z;
        const double c2 = s1 + g1 * z * c1;
        const double s2 = c2 + x1 * z * c1;
        return s2 + g2 * z * c2;
    };
    for (size_t gb = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gb < total; gb += (size_t)gridDim.x * blockDim.x) {
        const unsigned gline = fzh.div((unsigned)gb);
        const int k = (int)(gb - (size_t)gline * nzh);
        const unsigned ubox = a.fd_nl.div(gline);
        const unsigned line = gline - ubox * nlines;
        if (!a.sc[ubox].masked_live) continue;   // negligible masked content stays as it is
        const unsigned ui = a.fd_ny.div(line);
        const int i = (int)ui, j = (int)(line - ui * ny);
        if (a.g.mx[i] != 0.0 && a.g.my[j] != 0.0 && a.g.mz[k] != 0.0) continue;
        const size_t gi = (size_t)line * nzh + k;
        const size_t bo = (size_t)ubox * a.box_state;
        double2 X[6];
#pragma unroll
        for (int c = 0; c < 3; c++) X[c] = a.U[bo + (size_t)(a.VEL + c) * nc + gi];
        if (a.mhd)
#pragma unroll
            for (int c = 0; c < 3; c++) X[3 + c] = a.U[bo + (size_t)(a.MAG + c) * nc + gi];
        const double dt = a.sc[ubox].dt, nu = a.sc[ubox].nu, nu_m = a.sc[ubox].nu_m;
        const double kx = a.g.kx[i], ky = a.g.ky[j], kz = a.g.kz[k];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double cu = amp(-nu * k2 * dt);
        double2 Un[3];
#pragma unroll
        for (int c = 0; c < 3; c++) Un[c] = d2(cu * X[c].x, cu * X[c].y);
        if (a.clean) clean3(Un, kx, ky, kz);
#pragma unroll
        for (int c = 0; c < 3; c++) a.U[bo + (size_t)(a.VEL + c) * nc + gi] = Un[c];
        if (a.mhd) {
            const double cb = amp(-nu_m * k2 * dt);
#pragma unroll
            for (int c = 0; c < 3; c++) Un[c] = d2(cb * X[3 + c].x, cb * X[3 + c].y);
            if (a.clean) clean3(Un, kx, ky, kz);
#pragma unroll
            for (int c = 0; c < 3; c++) a.U[bo + (size_t)(a.MAG + c) * nc + gi] = Un[c];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_rkl_flux(const __grid_constant__ RklArgs a, double2* U, int vslot, FastDiv fzh,
                                                  FastDiv fny) {
    if (a.stage > a.sc->s_rkl) return;
    const double* cf = a.sc->rkl[a.stage];
    const size_t nc = a.g.nc;
    const int nzh = a.g.nzh, nzs = a.g.nzs;
    const C2<T>* nl = (const C2<T>*)a.nl;
    double2* Uc = U + (size_t)a.fields[vslot] * nc;
    const double shx = grid_shx(a.g);   // shearing box: the wavevector of the current remap clock
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const unsigned line = fzh.div((unsigned)gi);
        const int k = (int)(gi - (size_t)line * nzh);
        const unsigned ui = fny.div(line);
        const int i = (int)ui, j = (int)(line - ui * (unsigned)a.g.ny);
        double2 dU = d2(0.0, 0.0);
        if (a.g.mx[i] != 0.0 && a.g.my[j] != 0.0 && a.g.mz[k] != 0.0) {
            const size_t li = (size_t)line * nzs + k;
            const double2 q0 = to_d2(nl[li]), q1 = to_d2(nl[a.cs_nl + li]), q2 = to_d2(nl[2 * a.cs_nl + li]);
            const double kx = a.g.kx[i] + shx * a.g.ky[j], ky = a.g.ky[j], kz = a.g.kz[k];
            const double2 sq = d2(kx * q0.x + ky * q1.x + kz * q2.x, kx * q0.y + ky * q1.y + kz * q2.y);
            dU = d2(-sq.y, sq.x);   // i * mask * k.q
        }
        rkl_update(a, cf, (size_t)vslot * nc, gi, Uc, dU);
    }
}

}  // namespace spk
