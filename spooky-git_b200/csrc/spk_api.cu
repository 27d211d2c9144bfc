// spk_api.cu -- context, pipelines and the C ABI of include/spooky_b200.h.
//
// Reference = LorenzoLMP/spooky-git.  The host logic mirrors
// Supervisor/Fields/TimeStepping/RKLegendre; every step is recorded once
// into a CUDA graph (two graphs when RKL2 alternates before/after RK3) and
// replayed without host synchronisation.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/spooky_b200.h"
#include "spk_kernels.cuh"

#include "spk_kernels.cu"
#include "spk_pass2.cu"
#include "spk_closure.cu"
#include "spk_config.hpp"

using namespace spk;

static std::string g_create_error;

#define MAXT 256

struct spk_ctx {
    spk_params_t p;
    cudaStream_t stream;
    bool own_stream;
    bool fp32;
    int F, VX, VY, VZ, BX, BY, BZ, TH, VEL, MAG;
    int nx, ny, nz, nzh;
    size_t nc, nr;
    std::vector<double> kx, ky, kz, mx, my, mz;
    double kxmax, kymax, kzmax, kmax;
    int kz_keep;
    unsigned sts_mask;
    int nsts, sts_fields[8], sts_kind[8];
    bool sts_aniso, sts_iso, aniso_rhs;
    int rkl_smax;
    // device memory
    double* d_tab;                 // kx ky kz mx my mz
    void* d_tw;                    // twiddles x, y, z in pass precision
    FftPlan plan_x, plan_y, plan_z;
    double2 *U, *S;
    void *bufA, *bufB;
    int nbuf_ch;
    void *rA, *rB, *breal;
    double2 *Uc0, *Uc1, *dU0;
    DevScalars* sc;
    DevScalars* h_sc;              // pinned mirror
    double* d_sums;
    double* h_sums;
    DevGrid g;
    // pipeline layout
    int nin, nout, ch_u, ch_b, ch_th, ch_gx, ch_gy;
    int nin_base;                  // u, B, theta channels (no gradient channels)
    // learned closure: d/dx and d/dy channels of u [and B] (ncl_half each),
    // parameters on the device, Delta^2; closure_on once weights are set
    // deferred dealiased-out modes (HD/MHD RK3, no STS): kept x / y indices
    bool defer = false;
    int* d_keep = nullptr;
    int nkx = 0, nky = 0;
    bool trim_now = false;         // recording a step: the inverse passes may trim (DevScalars::masked_live)
    double stage_csh = 0.0;        // shearing box: the recorded RK stage's offset of the remap clock, in dt
    // schedule knobs picked by spk_autotune (0: the launchers' own choice)
    int tune_zl = 0;               // z pass: lines per CTA
    int tune_nst = 0;              // axis passes: pipeline stages
    int tune_kt = 0;               // axis passes of short axes: 2 = half-width tiles
    int tune_rhs = 0;              // RHS: CTAs per SM
    int ch_dx = -1, ch_dy = -1, ncl_half = 0;
    int ngrad = 0;                 // closure variant 2: gradient channels (9 or 18) from ch_dx
    double hp_k2 = 0.0;            // closure variant 2: small scales |k|^2 > hp_k2
    // shell spectra: bins (InputOutput / Wavevector, wavevector.cu:100-111)
    int nbins = 0;
    double deltak = 0.0;
    double* d_spec = nullptr;
    bool closure_on = false;
    float* d_cparams = nullptr;
    unsigned char* d_cimg = nullptr;   // variant 3: the packed BF16 network
    double delta2 = 0.0;
    int out_T, out_E, out_F, out_Q;
    // graphs
    cudaGraphExec_t gexec[2];
    bool have_graph[2];
    // graphs of steps on a caller's state array (spk_advance_fields), for the array last used
    cudaGraphExec_t fgexec[2];
    bool have_fgraph[2] = {false, false};
    const double2* fields_graph_ptr = nullptr;
    int h_step;
    std::string err;
    int sticky;
    long launches;                 // kernels issued (counted by the launch helpers)
    bool bad_job;                  // a pass could not be built (channel range, tensor map)
    const char* bad_why;
    const void* user_U;            // caller's state array during spk_compute_dfield
    bool dirty;                    // state set from outside: clean u, B before the next step
    int num_sms;
    // boxes of one geometry side by side (ensembles): U, S [nb][F][nc], pass
    // buffers [nb][nbuf_ch][ncs], DevScalars[nb] with each box's viscosities
    int nb = 1;
    std::vector<double> bnu, bnu_m, bnu_th;
    int kernels_per_step[2];
};

static int fail(spk_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg; else g_create_error = msg;
    return code;
}

#define CK(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return fail(c, SPK_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// buffer addressing
// ---------------------------------------------------------------------------
// Row length of the pass buffers (complex elements).  At least nzh, even
// (16-byte TMA strides); from 64 up, a multiple of 128 bytes, so that a
// 128-byte tile row never straddles DRAM bursts (rows of the x passes are far
// apart and share no sectors in L2).  The tensor maps keep nzh as the logical
// extent, so the padding is never read.
static int pass_row(int nzh, bool fp32) {
    if (nzh < 64) return nzh + (nzh & 1);
    return fp32 ? (nzh + 15) & ~15 : (nzh + 7) & ~7;
}
static size_t csize(const spk_ctx* c) { return c->fp32 ? sizeof(float2) : sizeof(double2); }
static size_t chan_bytes(const spk_ctx* c) { return c->g.ncs * csize(c); }
static int buf_channels(const spk_ctx* c, const void* base) {
    return (base == c->rA || base == c->rB) ? 3 : c->nbuf_ch;
}
// Channel ch of a pass buffer; channels outside the buffer give nullptr
// (add_job / zpass refuse null pointers) instead of addressing other memory.
static void* chan(const spk_ctx* c, void* base, int ch) {
    if (!base || ch < 0 || ch >= buf_channels(c, base)) return nullptr;
    return (char*)base + (size_t)ch * chan_bytes(c);
}

// True when [p, p + nch channels) lies inside one of the context's arrays.
static bool span_ok(const spk_ctx* c, const void* p, int nch, bool state) {
    if (!p || nch < 1) return false;
    const char* q = (const char*)p;
    const size_t cb = state ? c->nc * sizeof(double2) : chan_bytes(c);
    const size_t need = (size_t)nch * cb;
    auto inside = [&](const void* base, size_t bytes) {
        const char* b = (const char*)base;
        return b && q >= b && q + need <= b + bytes;
    };
    if (state) return inside(c->U, (size_t)c->F * c->nc * sizeof(double2)) ||
                      inside(c->user_U, (size_t)c->F * c->nc * sizeof(double2));
    return inside(c->bufA, (size_t)c->nbuf_ch * cb) || inside(c->bufB, (size_t)c->nbuf_ch * cb) ||
           inside(c->rA, 3 * cb) || inside(c->rB, 3 * cb);
}

// The array a channel pointer belongs to: (base, channels, channel index).
static bool locate(const spk_ctx* c, const void* p, bool state, const void** base, int* nchan, int* ch) {
    const char* q = (const char*)p;
    if (state) {
        const void* cands[2] = {c->U, c->user_U};
        for (const void* b : cands) {
            if (!b) continue;
            const size_t cb = c->nc * sizeof(double2);
            if (q >= (const char*)b && q < (const char*)b + (size_t)c->F * cb && (size_t)(q - (const char*)b) % cb == 0) {
                *base = b; *nchan = c->F * (b == c->U ? c->nb : 1); *ch = (int)((q - (const char*)b) / cb);
                return true;
            }
        }
        return false;
    }
    const void* cands[4] = {c->bufA, c->bufB, c->rA, c->rB};
    for (const void* b : cands) {
        if (!b) continue;
        const size_t cb = chan_bytes(c);
        if (cb == 0) return false;
        const int n = buf_channels(c, b);
        if (q >= (const char*)b && q < (const char*)b + (size_t)n * cb && (size_t)(q - (const char*)b) % cb == 0) {
            *base = b; *nchan = n * ((b == c->bufA || b == c->bufB) ? c->nb : 1); *ch = (int)((q - (const char*)b) / cb);
            return true;
        }
    }
    return false;
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

// 4-D tensor map [channel][x][y][k scalars] of a state array (FP64, rows of
// nzh complex) or a pass buffer (pass type, rows of nzs complex, logical
// extent nzh so that k >= nzh reads as zero), box = KT columns x box_rows
// positions along the axis.
static bool make_tmap(const spk_ctx* c, const void* base, int nchan, bool state, int axis, int kt, int box_rows,
                      CUtensorMap* tm) {
    if (!g_encode) return false;
    const bool f64 = state || !c->fp32;
    const size_t esz = f64 ? 8 : 4;
    const size_t row = state ? (size_t)c->nzh : (size_t)c->g.nzs;
    cuuint64_t dims[4] = {(cuuint64_t)(2 * c->nzh), (cuuint64_t)c->ny, (cuuint64_t)c->nx, (cuuint64_t)nchan};
    cuuint64_t strides[3] = {(cuuint64_t)(2 * row * esz), (cuuint64_t)(2 * row * esz * c->ny),
                             (cuuint64_t)(2 * row * esz * c->ny * c->nx)};
    cuuint32_t box[4];
    if (axis == 0) { box[0] = 2 * kt; box[1] = 1; box[2] = box_rows; box[3] = 1; }
    else           { box[0] = 2 * kt; box[1] = box_rows; box[2] = 1; box[3] = 1; }
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = g_encode(tm, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                          const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

static AxisArgs axis_args(spk_ctx* c, int ax) {
    AxisArgs a;
    memset(&a, 0, sizeof(a));
    a.g = c->g;
    a.g.csh = c->stage_csh;
    a.plan = ax == 0 ? c->plan_x : c->plan_y;
    a.axis = ax;
    a.kcols = c->nzh;
    a.scale = 1.0;
    a.nb = c->nb;
    a.out_box_ch = c->nbuf_ch;
    a.scs = c->sc;
    return a;
}

// ---------------------------------------------------------------------------
// FFT twiddles W_N^k in long double (rounded once to the pass precision).
// ---------------------------------------------------------------------------
static void twiddles(int n, std::vector<double>& out) {
    const long double PI = 3.141592653589793238462643383279502884L;
    out.resize(2 * (size_t)n);
    for (int k = 0; k < n; k++) {
        long double a = 2.0L * PI * (long double)k / (long double)n;
        out[2 * k] = (double)cosl(a);
        out[2 * k + 1] = -(double)sinl(a);
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------

struct AxisCfg { int kt; int nthr; size_t smem; };

// Tile width of a strided-axis pass: the host mirror of axis_kt<T, N, CONV>
// (KT columns x TPC threads = 256 threads, KT <= 64; an FP64 input tile in
// the FP32 form is half as wide).
static AxisCfg axis_cfg(const spk_ctx* c, int N, bool state_in) {
    AxisCfg a;
    const RegFftGeom g = regfft_geom(N, c->fp32);
    const int full = std::min(64, 256 / g.TPC);
    const int cols = std::max(pow2_ceil(N / 2 + 1), 32 / g.TPC);   // short axes: a cubic box's kz columns
    int kt = (N < 64 && cols < full) ? cols : full;
    if (c->fp32 && state_in && kt == full && kt > 2) kt /= 2;
    kt = std::max(kt, 2);
    // the autotuner's half tiles of short axes (axis_half_ok)
    if (c->tune_kt == 2 && N <= 64 && kt / 2 >= 2 && (kt / 2) * g.TPC >= 32) kt /= 2;
    a.kt = kt;
    a.nthr = kt * g.TPC;
    a.smem = 0;
    return a;
}


// The dynamic shared-memory cap of a pass kernel: the opt-in maximum, set
// alike by every launch.  One instantiation serves contexts and ensemble
// groups with different tile sizes, and a cap set to one launch's size would
// be too small for a recorded launch of another (a kernel node launched on
// its own, as a profiler's replay does).  Occupancy follows each launch's
// own size.
template <typename K> static void allow_full_smem(K* kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

template <typename T, int N, int DIR, bool CONV, bool DEF, int KTD>
static void launch_axis_kt(spk_ctx* c, AxisArgs& a, long total) {
    constexpr int KT = axis_kt<T, N, CONV, KTD>();
    const int nthr = KT * RegFft<T, N>::TPC;
    const size_t in_elem = CONV ? sizeof(double2) : sizeof(C2<T>);
    const size_t stage = (((size_t)N * KT * in_elem) + 127) & ~(size_t)127;
    // barriers + stages + exchange + twiddles + wavenumbers + row mask (+ alignment)
    const size_t fixed = 256 + (size_t)N * KT * sizeof(C2<T>) + (size_t)RegFft<T, N>::TWN * sizeof(C2<T>) +
                         (size_t)N * sizeof(T) + N + 1024 + 16;   // ... + row mask + outer mask (<= 1024)
    // stages: as many as keep axis_minb CTAs per SM (228 KB per SM, 1 KB
    // reserved per CTA): three CTAs of <= 75 KB with 1..4 stages, or two of
    // <= 113 KB with 2..4 (also when one stage does not fit the three-CTA size)
    long nst = ((long)(75 * 1024) - (long)fixed) / (long)stage;
    if (axis_minb<T, N>() == 3 && nst >= 1) {
        a.nst = (int)std::min<long>(4, nst);
    } else {
        nst = ((long)(113 * 1024) - (long)fixed) / (long)stage;
        a.nst = (int)std::max<long>(2, std::min<long>(4, nst));
    }
    if (nthr < 256) {
        // narrow tiles (128 threads): 4 CTAs per SM with fewer stages each keep
        // as many loads in flight as 2 CTAs with more, with twice the warps
        const long nst4 = ((long)(56 * 1024) - (long)fixed) / (long)stage;
        if (nst4 >= 1) a.nst = (int)std::min<long>(4, nst4);
    }
    if (c->tune_nst >= 1 && c->tune_nst <= 4 && fixed + (size_t)c->tune_nst * stage <= (size_t)227 * 1024)
        a.nst = c->tune_nst;
    const size_t smem = fixed + (size_t)a.nst * stage;
    allow_full_smem(k_axis2<T, N, DIR, CONV, DEF, KTD>);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_axis2<T, N, DIR, CONV, DEF, KTD>, nthr, smem);
    const int grid = (int)std::min<long>(total, (long)c->num_sms * std::max(per_sm, 1));
    c->launches++;
    k_axis2<T, N, DIR, CONV, DEF, KTD><<<grid, nthr, smem, c->stream>>>(a);
}

// the tile width the arguments carry (axis_cfg) picks the instantiation
template <typename T, int N, int DIR, bool CONV, bool DEF = false>
static void launch_axis_ln(spk_ctx* c, AxisArgs& a, long total) {
    if (a.kt == axis_kt<T, N, CONV, 1>()) { launch_axis_kt<T, N, DIR, CONV, DEF, 1>(c, a, total); return; }
    if constexpr (axis_half_ok<T, N, CONV>()) {
        if (a.kt == axis_kt<T, N, CONV, 2>()) { launch_axis_kt<T, N, DIR, CONV, DEF, 2>(c, a, total); return; }
    }
    c->err = "internal: axis tile width mismatch";
    c->sticky = SPK_ERR_ARG;
}

template <typename T, int N, int DIR>
static void launch_axis_conv(spk_ctx* c, AxisArgs& a, long total) {
    if constexpr (DIR > 0) {
        if (a.defer_stage) {   // x inverse of a deferred stage: state input
            if constexpr (sizeof(T) == 4) {
                if (a.convert) { launch_axis_ln<T, N, DIR, true, true>(c, a, total); return; }
            } else {
                launch_axis_ln<T, N, DIR, false, true>(c, a, total);
                return;
            }
        }
    }
    if constexpr (sizeof(T) == 4 && DIR > 0) {
        if (a.convert) { launch_axis_ln<T, N, DIR, true>(c, a, total); return; }
    }
    launch_axis_ln<T, N, DIR, false>(c, a, total);
}

// Every transform length the register FFT covers (2^k and 3*2^k).
#define SPK_FOR_EACH_LENGTH(X) \
    X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(6) X(12) X(24) X(48) X(96) X(192) X(384) X(768)

template <typename T, int DIR>
static void launch_axis_dir(spk_ctx* c, AxisArgs& a, long total) {
    switch (a.plan.n) {
#define SPK_AXIS_CASE(n) case n: launch_axis_conv<T, n, DIR>(c, a, total); break;
        SPK_FOR_EACH_LENGTH(SPK_AXIS_CASE)
#undef SPK_AXIS_CASE
        default: c->err = "internal: unsupported axis length"; c->sticky = SPK_ERR_UNSUPPORTED; break;
    }
}

template <typename T>
static void launch_axis(spk_ctx* c, AxisArgs& a, int dir) {
    const int nouter = a.axis == 0 ? c->ny : c->nx;
    const int nkb = (a.kcols + a.kt - 1) / a.kt;
    const long total = (long)a.njobs * a.nb * nouter * nkb;
    if (total <= 0) return;
    a.err = &c->sc->err;
    a.fd_kb = FastDiv::make((unsigned)nkb);
    a.fd_box = FastDiv::make((unsigned)(nouter * nkb));
    a.fd_job = FastDiv::make((unsigned)(a.nb * nouter * nkb));
    if (a.outer_filter && a.axis == 0 && !a.trim && c->d_keep) {
        // outer-filtered x forward: walk the kept ky rows only
        a.tr_always = 1;
        a.tr_nkb = nkb;
        a.tr_nouter = c->nky;
        a.tr_outer = c->d_keep + c->nkx;
        a.tr_fd_kb = FastDiv::make((unsigned)a.tr_nkb);
        a.tr_fd_box = FastDiv::make((unsigned)(a.tr_nouter * a.tr_nkb));
        a.tr_fd_job = FastDiv::make((unsigned)(a.nb * a.tr_nouter * a.tr_nkb));
    }
    if (a.trim) {
        // kept tiles of a trimmed single-box pass (used when the state has no masked content)
        a.tr_nkb = std::max(1, (c->kz_keep + a.kt - 1) / a.kt);
        a.tr_nouter = a.trim == 1 ? c->nky : nouter;
        a.tr_outer = c->d_keep + c->nkx;   // kept y indices
        a.tr_fd_kb = FastDiv::make((unsigned)a.tr_nkb);
        a.tr_fd_box = FastDiv::make((unsigned)(a.tr_nouter * a.tr_nkb));
        a.tr_fd_job = FastDiv::make((unsigned)(a.nb * a.tr_nouter * a.tr_nkb));
    }
    if (dir > 0) launch_axis_dir<T, +1>(c, a, total);
    else launch_axis_dir<T, -1>(c, a, total);
}

static void axis(spk_ctx* c, AxisArgs& a, int dir) {
    if (c->bad_job) {
        char buf[256];
        snprintf(buf, sizeof(buf), " (axis %d, jobs %d, nbuf_ch %d, ncs %zu, nc %zu)", a.axis, a.njobs, c->nbuf_ch,
                 (size_t)c->g.ncs, (size_t)c->nc);
        c->err = std::string("internal: ") + c->bad_why + buf;
        c->sticky = SPK_ERR_ARG;
        return;
    }
    if (a.njobs == 0) return;
    if (a.row_filter && dir > 0) {   // the three-CTA k_axis2 filters the rows of forward passes only
        c->err = "internal: row filter on an inverse axis pass";
        c->sticky = SPK_ERR_ARG;
        return;
    }
    if (c->fp32) launch_axis<float>(c, a, dir);
    else launch_axis<double>(c, a, dir);
}

template <typename T, int N>
static void launch_zpass_ln(spk_ctx* c, ZArgs& z, int nin_all) {
    const int nthr = 128;
    const int slots = std::max(1, nthr / RegFft<T, N>::TPC);
    const long nlines = (long)c->nx * c->ny;
    const int npin = (nin_all + 1) / 2, npout = (z.nout + 1) / 2;
    const int gen = z.closure == 3 ? 3 : (z.closure ? 2 : ((z.derive_gz != 0 || z.mode == ZM_TO_REAL || z.shear_part) ? 1 : 0));
    const int max_ctas = gen == 0 ? (sizeof(T) == 4 ? 6 : 5) : 4;   // the kernel's launch bounds
    auto need = [&](int lines) {
        return zsmem_layout(N, RegFft<T, N>::TWN, (int)sizeof(C2<T>), z.nin, nin_all, npout, lines, c->g.nzs,
                            slots, z.closure == 3 ? C3_ZBYTES / 4 : (z.closure ? CL_NP : 0),
                            zpass_alias(gen, RegFft<T, N>::NS, npin, npout, lines, slots),
                            (gen == 1 && z.load_breal && zpass_stage_b<T, N>()) ? 3 : 0).total;
    };
    // lines per CTA: best (busy transform slots) x (resident CTAs per SM, <= 4)
    auto rounds = [&](long n) { return (n + slots - 1) / slots; };
    int L = 1;
    double best = -1.0;
    for (int cand = 1; cand <= 64 && cand <= nlines; cand *= 2) {
        if (c->nb > 1 && nlines % cand != 0) break;   // a CTA's lines stay inside one box
        const size_t sm = need(cand);
        if (sm > (size_t)227 * 1024) break;
        const long work = (long)(npin + npout) * cand;
        const long cap = (rounds((long)npin * cand) + rounds((long)npout * cand)) * slots;
        const double util = (double)work / (double)std::max<long>(cap, 1);
        const int ctas = (int)std::min<size_t>((size_t)max_ctas, (size_t)(233472 / (sm + 1024)));
        const double score = util * ctas;
        if (score >= best) { best = score; L = cand; }
    }
    if (c->tune_zl > 0 && c->tune_zl <= nlines && need(c->tune_zl) <= (size_t)227 * 1024 &&
        (c->nb == 1 || nlines % c->tune_zl == 0))
        L = c->tune_zl;
    const size_t smem = need(L);
    if (smem > (size_t)227 * 1024) {
        c->err = "internal: z pass tile exceeds shared memory";
        c->sticky = SPK_ERR_UNSUPPORTED;
        return;
    }
    z.lines = L;
    const int nblk = (int)(((nlines + L - 1) / L) * c->nb);
    c->launches++;
    if (z.closure == 3) {
        allow_full_smem(k_zpass2<T, N, 3>);
        k_zpass2<T, N, 3><<<nblk, nthr, smem, c->stream>>>(z);
    } else if (z.closure) {
        allow_full_smem(k_zpass2<T, N, 2>);
        k_zpass2<T, N, 2><<<nblk, nthr, smem, c->stream>>>(z);
    } else if (z.derive_gz != 0 || z.mode == ZM_TO_REAL || z.shear_part) {
        allow_full_smem(k_zpass2<T, N, 1>);
        k_zpass2<T, N, 1><<<nblk, nthr, smem, c->stream>>>(z);
    } else {
        allow_full_smem(k_zpass2<T, N, 0>);
        k_zpass2<T, N, 0><<<nblk, nthr, smem, c->stream>>>(z);
    }
}

template <typename T>
static void launch_zpass(spk_ctx* c, ZArgs& z, int nin_all) {
    switch (c->nz) {
#define SPK_Z_CASE(n) case n: launch_zpass_ln<T, n>(c, z, nin_all); break;
        SPK_FOR_EACH_LENGTH(SPK_Z_CASE)
#undef SPK_Z_CASE
        default: c->err = "internal: unsupported z length"; c->sticky = SPK_ERR_UNSUPPORTED; break;
    }
}

static void zpass(spk_ctx* c, ZArgs& z) {
    if (!span_ok(c, z.in, std::max(z.nin, 1), false) || (z.nout > 0 && !span_ok(c, z.out, z.nout, false)) ||
        ((z.store_breal || z.load_breal) && !c->breal)) {
        c->err = "internal: a z pass addressed channels outside its buffers";
        c->sticky = SPK_ERR_ARG;
        return;
    }
    const int nin_all = z.nin + (z.derive_gz == 1 ? 1 : 0) + z.zder_n;
    if (c->fp32) launch_zpass<float>(c, z, nin_all);
    else launch_zpass<double>(c, z, nin_all);
}

static int ew_blocks(size_t n) {
    return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// ---------------------------------------------------------------------------
// argument builders
// ---------------------------------------------------------------------------
// nch consecutive channels from `in` (state array or pass buffer) to `out`,
// one job (and one tensor map) per channel.
static void add_job(spk_ctx* c, AxisArgs& a, const void* in, void* out, int nch, int in_state, int deriv, int clean) {
    (void)clean;
    const void* base;
    int nchan, ch0;
    const char* why = nullptr;
    if (!span_ok(c, in, nch, in_state != 0)) why = "pass job input outside its array";
    else if (!span_ok(c, out, nch, false)) why = "pass job output outside its buffer";
    else if (a.njobs + nch > SPK_MAXJOBS) why = "too many pass jobs";
    else if (!locate(c, in, in_state != 0, &base, &nchan, &ch0)) why = "pass job input not at a channel boundary";
    if (why) {
        c->bad_job = true;
        c->bad_why = why;
        return;
    }
    const int N = a.plan.n;
    const AxisCfg cf = axis_cfg(c, N, in_state != 0);
    if (a.njobs > 0 && a.kt != cf.kt) { c->bad_job = true; c->bad_why = "jobs of one pass need one tile width"; return; }
    a.kt = cf.kt;
    a.box_rows = N;                               // rows per TMA box: a divisor of N, <= 256
    while (a.box_rows > 256) {
        int d = 256;
        while (N % d) d--;
        a.box_rows = d;
    }
    if (in_state && c->fp32) a.convert = 1;
    a.in_box_ch = in_state ? c->F : buf_channels(c, base);
    if (c->nb > 1 && (base == c->rA || base == c->rB || base == c->user_U)) {
        c->bad_job = true;
        c->bad_why = "a single-box buffer in a multi-box pass";
        return;
    }
    for (int q = 0; q < nch; q++) {
        AxisJob& j = a.job[a.njobs++];
        if (!make_tmap(c, base, nchan, in_state != 0, a.axis, a.kt, a.box_rows, &j.tm)) {
            c->bad_job = true;
            c->bad_why = "cuTensorMapEncodeTiled rejected a pass tensor map";
            return;
        }
        j.out = (char*)out + (size_t)q * chan_bytes(c);
        j.ch = ch0 + q;
        j.in_state = in_state;
        j.deriv = deriv;
    }
}

// first inverse pass over the state: fields in order.  stage: the RK3 stage
// (1 or 2 with deferred masked modes scales those modes to the stage's value)
static void pass_x_inverse(spk_ctx* c, const double2* U, bool with_gx, int stage = 0) {
    AxisArgs a = axis_args(c, 0);
    a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);   // scaleKernel factor
    a.defer_stage = (c->defer && c->d_keep && U == c->U && (stage == 1 || stage == 2)) ? stage : 0;
    a.trim = (c->trim_now && U == c->U) ? 1 : 0;
    auto mark = [&](int first, int grp) {
        for (int q = first; q < a.njobs; q++) a.job[q].defer_grp = grp;
    };
    if (c->p.incompressible) { const int j0 = a.njobs; add_job(c, a, U + (size_t)c->VEL * c->nc, chan(c, c->bufA, c->ch_u), 3, 1, 0, 0); mark(j0, 1); }
    if (c->p.mhd) { const int j0 = a.njobs; add_job(c, a, U + (size_t)c->MAG * c->nc, chan(c, c->bufA, c->ch_b), 3, 1, 0, 0); mark(j0, 2); }
    if (c->p.boussinesq) {
        add_job(c, a, U + (size_t)c->TH * c->nc, chan(c, c->bufA, c->ch_th), 1, 1, 0, 0);
        if (with_gx && c->aniso_rhs) add_job(c, a, U + (size_t)c->TH * c->nc, chan(c, c->bufA, c->ch_gx), 1, 1, 1, 0);
    }
    if (with_gx && c->closure_on && c->ngrad == 0) {
        int j0 = a.njobs;
        add_job(c, a, U + (size_t)c->VEL * c->nc, chan(c, c->bufA, c->ch_dx), 3, 1, 1, 0);
        mark(j0, 1);
        if (c->p.mhd) {
            j0 = a.njobs;
            add_job(c, a, U + (size_t)c->MAG * c->nc, chan(c, c->bufA, c->ch_dx + 3), 3, 1, 1, 0);
            mark(j0, 2);
        }
    }
    // closure variant 2: d/dx_j of the small scales of u (then B), channel ch_dx + 3 j + i
    auto grad_jobs = [&](AxisArgs& g, int field, int ch0, int grp) {
        g.hp_k2 = c->hp_k2;
        for (int j = 0; j < 3; j++) {
            const int j0 = g.njobs;
            add_job(c, g, U + (size_t)field * c->nc, chan(c, c->bufA, ch0 + 3 * j), 3, 1, j + 1, 0);
            for (int q = j0; q < g.njobs; q++) { g.job[q].defer_grp = grp; g.job[q].hp = 1; }
        }
    };
    const bool grad9 = with_gx && c->closure_on && c->ngrad > 0;
    if (grad9) grad_jobs(a, c->VEL, c->ch_dx, 1);
    axis(c, a, +1);
    if (grad9 && c->p.mhd) {
        AxisArgs b = axis_args(c, 0);
        b.scale = a.scale;
        b.defer_stage = a.defer_stage;
        b.trim = a.trim;
        grad_jobs(b, c->MAG, c->ch_dx + 9, 2);
        axis(c, b, +1);
    }
}

static void pass_y_inverse(spk_ctx* c, bool with_g) {
    AxisArgs a = axis_args(c, 1);
    a.trim = c->trim_now ? 2 : 0;
    if (with_g && c->aniso_rhs) {
        // u, B, theta and d/dx theta one to one; d/dy theta from theta
        add_job(c, a, c->bufA, c->bufB, c->ch_gx + 1, 0, 0, 0);
        add_job(c, a, chan(c, c->bufA, c->ch_th), chan(c, c->bufB, c->ch_gy), 1, 0, 1, 0);
    } else if (with_g && c->closure_on && c->ngrad > 0) {
        // variant 2: every channel one to one, in launches of at most SPK_MAXJOBS jobs
        const int n = c->nin_base + c->ngrad;
        for (int c0 = 0; c0 < n; c0 += SPK_MAXJOBS) {
            AxisArgs b = axis_args(c, 1);
            b.trim = a.trim;
            const int m = std::min(SPK_MAXJOBS, n - c0);
            add_job(c, b, chan(c, c->bufA, c0), chan(c, c->bufB, c0), m, 0, 0, 0);
            axis(c, b, +1);
        }
        return;
    } else if (with_g && c->closure_on) {
        // u, B and their d/dx one to one; then d/dy of u, B (a second launch:
        // the jobs of one launch are capped)
        add_job(c, a, c->bufA, c->bufB, c->ch_dx + c->ncl_half, 0, 0, 0);
        axis(c, a, +1);
        AxisArgs b = axis_args(c, 1);
        b.trim = a.trim;
        add_job(c, b, chan(c, c->bufA, c->ch_u), chan(c, c->bufB, c->ch_dy), c->ncl_half, 0, 1, 0);
        axis(c, b, +1);
        return;
    } else {
        add_job(c, a, c->bufA, c->bufB, c->nin_base, 0, 0, 0);
    }
    axis(c, a, +1);
}

static ZArgs z_args(spk_ctx* c) {
    ZArgs z;
    memset(&z, 0, sizeof(z));
    z.g = c->g;
    z.plan = c->plan_z;
    z.in = c->bufB; z.cs_in = c->g.ncs;
    z.out = c->bufA; z.cs_out = c->g.ncs;
    z.ch_u = z.ch_b = z.ch_th = z.ch_gx = z.ch_gy = -1;
    z.maxbits = c->sc->maxbits;
    z.nonfinite = &c->sc->nonfinite;
    z.err = &c->sc->err;
    z.breal = c->breal;
    z.sd = c->p.strat_direction;
    z.chi = 1.0 / c->p.reynolds_ani;
    z.omegaT2 = c->p.OmegaT2;
    z.fd_nz = FastDiv::make((unsigned)c->nz);
    z.nb = c->nb;
    z.in_box = z.out_box = (size_t)c->nbuf_ch * c->g.ncs;
    z.scs = c->sc;
    return z;
}

static void set_inputs(spk_ctx* c, ZArgs& z, bool with_g) {
    z.nin = c->nin_base;
    z.ch_u = c->ch_u; z.ch_b = c->ch_b; z.ch_th = c->ch_th;
    if (with_g && c->aniso_rhs) { z.nin += 2; z.ch_gx = c->ch_gx; z.ch_gy = c->ch_gy; z.derive_gz = 1; }
    if (with_g && c->closure_on) {
        z.closure = c->p.closure == 3 ? 3 : 1;
        z.ch_dx = c->ch_dx;
        z.cparams = c->p.closure == 3 ? (const float*)c->d_cimg : c->d_cparams;
        z.delta2 = (float)c->delta2;
        if (c->ngrad > 0) {
            z.nin += c->ngrad;
            z.cl_grad9 = 1;
        } else {
            z.nin += 2 * c->ncl_half;
            z.ch_dy = c->ch_dy;
            z.zder_n = c->ncl_half;
            for (int d = 0; d < c->ncl_half; d++) z.zder_src[d] = c->ch_u + d;
        }
    }
}

static void pass_z_products(spk_ctx* c, bool do_max) {
    ZArgs z = z_args(c);
    z.mode = ZM_PRODUCTS;
    z.trim = c->trim_now ? 1 : 0;
    set_inputs(c, z, true);
    z.nout = c->nout;
    z.hydro = 1;
    z.mhd = c->p.mhd; z.bous = c->p.boussinesq; z.aniso = c->aniso_rhs ? 1 : 0;
    z.do_max = do_max ? 1 : 0;
    zpass(c, z);
}

static void pass_z_inverse_only(spk_ctx* c, bool do_max, bool store_b) {
    ZArgs z = z_args(c);
    z.mode = ZM_INVERSE_ONLY;
    set_inputs(c, z, false);
    z.nout = 0;
    z.do_max = do_max ? 1 : 0;
    z.store_breal = store_b ? 1 : 0;
    zpass(c, z);
}

static void pass_y_forward(spk_ctx* c, int nch, void* in, void* out) {
    AxisArgs a = axis_args(c, 1);
    a.kcols = c->kz_keep;
    a.row_filter = 1;
    add_job(c, a, in, out, nch, 0, 0, 0);
    if (a.kcols > 0) axis(c, a, -1);
}

// x-forward pass of the products (bufB -> bufA): kept ky rows in, kept kx
// rows out, kz < kz_keep.
static void pass_x_forward(spk_ctx* c) {
    AxisArgs a = axis_args(c, 0);
    a.kcols = c->kz_keep;
    a.row_filter = 1;
    a.outer_filter = 1;
    add_job(c, a, c->bufB, c->bufA, c->nout, 0, 0, 0);
    if (a.kcols > 0) axis(c, a, -1);
}

// elementwise RHS + Leray + time update of every mode
static void rhs(spk_ctx* c, XfArgs& x) {
    const FastDiv fz = FastDiv::make((unsigned)c->nzh);
    // 128-thread CTAs, three per SM: every load of a mode is issued up front
    const size_t modes = x.defer ? (size_t)x.nkx * x.nky * c->kz_keep : c->nc;
    const size_t per_sm = c->tune_rhs > 0 ? (size_t)c->tune_rhs : 24;
    const int grid = (int)std::min<size_t>((modes * c->nb + 127) / 128, (size_t)c->num_sms * per_sm);
    c->launches++;
    if (c->fp32 && !c->p.boussinesq) k_rhs<float, 4><<<grid, 128, 0, c->stream>>>(x, fz);
    else if (c->fp32) k_rhs<float, 3><<<grid, 128, 0, c->stream>>>(x, fz);
    else k_rhs<double, 3><<<grid, 128, 0, c->stream>>>(x, fz);
    if (x.defer && x.mode == XM_RK2) {
        // the step's masked modes, once
        c->launches++;
        k_masked_rk<<<ew_blocks(c->nc * c->nb), 256, 0, c->stream>>>(x, fz);
    }
}

static void xfwd(spk_ctx* c, XfArgs& x) {
    pass_x_forward(c);
    rhs(c, x);
}

static XfArgs xf_args(spk_ctx* c, double2* U, int mode, bool clean) {
    XfArgs x;
    memset(&x, 0, sizeof(x));
    x.g = c->g;
    x.g.csh = c->stage_csh;
    x.plan = c->plan_x;
    x.nl = c->bufA; x.cs_nl = c->g.ncs;   // products after the x-forward pass
    x.fd_ny = FastDiv::make((unsigned)c->ny);
    x.fd_nl = FastDiv::make((unsigned)(c->nx * c->ny));
    x.nb = c->nb;
    x.box_state = (size_t)c->F * c->nc;
    x.box_nl = (size_t)c->nbuf_ch * c->g.ncs;
    x.nl_T = c->out_T; x.nl_E = c->out_E; x.nl_F = c->out_F; x.nl_Q = c->out_Q;
    x.U = U; x.S = c->S; x.out = nullptr;
    x.F = c->F; x.VEL = c->VEL; x.MAG = c->MAG; x.TH = c->TH;
    x.incompressible = c->p.incompressible; x.mhd = c->p.mhd; x.bous = c->p.boussinesq;
    x.heat = c->p.heat_equation; x.strat = c->p.stratification; x.sd = c->p.strat_direction;
    x.aniso_rhs = c->aniso_rhs ? 1 : 0;
    x.sts_mask = c->sts_mask;
    x.nu = c->p.nu; x.nu_m = c->p.nu_m; x.nu_th = c->p.nu_th; x.N2 = c->p.N2;
    x.mode = mode; x.clean = clean ? 1 : 0;
    x.sc = c->sc;
    x.rotating = c->p.rotating; x.omega = c->p.omega;
    x.defer = c->defer && c->d_keep && (mode == XM_RK0 || mode == XM_RK1 || mode == XM_RK2);
    if (x.defer) {
        x.kxi = c->d_keep; x.kyi = c->d_keep + c->nkx;
        x.nkx = c->nkx; x.nky = c->nky;
        x.fd_kzk = FastDiv::make((unsigned)c->kz_keep);
        x.fd_nky = FastDiv::make((unsigned)c->nky);
        x.fd_nkx = FastDiv::make((unsigned)c->nkx);
    }
    return x;
}

static DtArgs dt_args(spk_ctx* c, bool advance) {
    DtArgs d;
    memset(&d, 0, sizeof(d));
    const spk_params_t& p = c->p;
    d.incompressible = p.incompressible; d.heat = p.heat_equation; d.mhd = p.mhd; d.bous = p.boussinesq;
    d.aniso = p.anisotropic_diffusion; d.sts = p.supertimestepping && c->nsts > 0; d.with_fixed = p.fixed_dt > 0.0;
    d.kxmax = c->kxmax; d.kymax = c->kymax; d.kzmax = c->kzmax;
    d.nu = p.nu; d.nu_m = p.nu_m; d.nu_th = p.nu_th; d.reynolds_ani = p.reynolds_ani; d.N2 = p.N2; d.OmegaT2 = p.OmegaT2;
    d.cfl = p.cfl; d.cfl_par = p.cfl_par; d.cfl_sts = p.cfl_sts; d.safety_source = p.safety_source; d.safety_sts = p.safety_sts;
    d.t_final = p.t_final; d.toutput_flow = p.toutput_flow; d.fixed_dt = p.fixed_dt;
    d.sts_pos_mask = c->sts_mask;
    d.VX = c->VX; d.VY = c->VY; d.VZ = c->VZ; d.BX = c->BX; d.BY = c->BY; d.BZ = c->BZ; d.TH = c->TH;
    d.advance = advance ? 1 : 0;
    d.rkl_smax = c->rkl_smax;
    d.sts_alg = p.sts_algorithm;
    d.closure = c->closure_on ? 1 : 0;
    d.shearing = p.shearing; d.rotating = p.rotating; d.shear = p.shear; d.omega = p.omega;
    return d;
}

// ---------------------------------------------------------------------------
// Super-time-stepping cycle (RKLegendre::compute_cycle, rkl.cu:185-199:
// STS, RKL1 or RKL2); stages beyond the device-computed count exit
// immediately.
// ---------------------------------------------------------------------------
static RklArgs rkl_args(spk_ctx* c, int stage) {
    RklArgs r;
    memset(&r, 0, sizeof(r));
    r.g = c->g;
    r.plan = c->plan_x;
    r.nl = c->rB; r.cs_nl = c->g.ncs;
    r.Uc0 = c->Uc0; r.Uc1 = c->Uc1; r.dU0 = c->dU0;
    r.stage = stage;
    r.sts_alg = c->p.sts_algorithm;
    r.nsts = c->nsts;
    for (int v = 0; v < c->nsts; v++) { r.fields[v] = c->sts_fields[v]; r.kind[v] = c->sts_kind[v]; }
    r.nu = c->p.nu; r.nu_m = c->p.nu_m; r.nu_th = c->p.nu_th;
    r.sc = c->sc;
    return r;
}

static void record_rkl_cycle(spk_ctx* c) {
    for (int st = 1; st <= c->rkl_smax; st++) {
        if (c->sts_iso) {
            RklArgs r = rkl_args(c, st);
            c->launches++;
            k_rkl_spectral<<<ew_blocks(c->nc), 256, 0, c->stream>>>(r, c->U);
        }
        if (c->sts_aniso) {
            // theta and i*kx*theta, x inverse
            AxisArgs a = axis_args(c, 0);
            a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
            a.gate = c->sc; a.gate_stage = st;
            add_job(c, a, c->U + (size_t)c->TH * c->nc, chan(c, c->rA, 0), 1, 1, 0, 0);
            add_job(c, a, c->U + (size_t)c->TH * c->nc, chan(c, c->rA, 1), 1, 1, 1, 0);
            axis(c, a, +1);
            // y inverse: theta (for i*kz theta), i*ky theta, i*kx theta
            AxisArgs b = axis_args(c, 1);
            b.gate = c->sc; b.gate_stage = st;
            add_job(c, b, chan(c, c->rA, 0), chan(c, c->rB, 0), 1, 0, 0, 0);
            add_job(c, b, chan(c, c->rA, 0), chan(c, c->rB, 1), 1, 0, 1, 0);
            add_job(c, b, chan(c, c->rA, 1), chan(c, c->rB, 2), 1, 0, 0, 0);
            axis(c, b, +1);
            // z: gradient, real B, heat flux, R2C
            ZArgs z = z_args(c);
            z.gate = c->sc; z.gate_stage = st;
            z.mode = ZM_RKL_FLUX;
            z.in = c->rB; z.out = c->rA;
            z.nin = 3; z.ch_th = 0; z.ch_gy = 1; z.ch_gx = 2; z.derive_gz = 2;
            z.load_breal = 1; z.aniso = 1; z.nout = 3;
            zpass(c, z);
            AxisArgs f = axis_args(c, 1);
            f.gate = c->sc; f.gate_stage = st;
            f.kcols = c->kz_keep; f.row_filter = 1;
            add_job(c, f, c->rA, c->rB, 3, 0, 0, 0);
            if (f.kcols > 0) axis(c, f, -1);
            // x forward of the flux (kept ky rows in, kept kx rows out)
            AxisArgs x = axis_args(c, 0);
            x.gate = c->sc; x.gate_stage = st;
            x.kcols = c->kz_keep; x.row_filter = 1; x.outer_filter = 1;
            add_job(c, x, c->rB, c->rA, 3, 0, 0, 0);
            if (x.kcols > 0) axis(c, x, -1);
            RklArgs r = rkl_args(c, st);
            r.nl = c->rA;
            int vslot = 0;
            for (int v = 0; v < c->nsts; v++) if (c->sts_kind[v] == 3) vslot = v;
            const FastDiv fz = FastDiv::make((unsigned)c->nzh);
            c->launches++;
            if (c->fp32) k_rkl_flux<float><<<ew_blocks(c->nc), 256, 0, c->stream>>>(r, c->U, vslot, fz, FastDiv::make((unsigned)c->ny));
            else k_rkl_flux<double><<<ew_blocks(c->nc), 256, 0, c->stream>>>(r, c->U, vslot, fz, FastDiv::make((unsigned)c->ny));
        }
    }
}

// real-space B of the current state for the anisotropic STS flux
static void record_breal(spk_ctx* c) {
    AxisArgs a = axis_args(c, 0);
    a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
    add_job(c, a, c->U + (size_t)c->MAG * c->nc, chan(c, c->bufA, c->ch_b), 3, 1, 0, 0);
    axis(c, a, +1);
    AxisArgs b = axis_args(c, 1);
    add_job(c, b, chan(c, c->bufA, c->ch_b), chan(c, c->bufB, c->ch_b), 3, 0, 0, 0);
    axis(c, b, +1);
    ZArgs z = z_args(c);
    z.mode = ZM_INVERSE_ONLY;
    z.nin = c->ch_b + 3;   // channels before B are unused zeros of the pair layout
    z.ch_b = c->ch_b;
    z.store_breal = 1;
    zpass(c, z);
}

// ---------------------------------------------------------------------------
// one main-loop iteration (CleanFieldDivergence + HydroMHDAdvance)
// ---------------------------------------------------------------------------
// rk_only: TimeStepping::RungeKutta3 (or ForwardEuler) alone, with the dt
// already in the device scalars: no dt reduction, no super-time-stepping,
// no divergence cleaning of the result.
static void record_step_body(spk_ctx* c, int parity, bool rk_only = false);
static void launch_clean(spk_ctx* c);
// The inverse passes of a recorded step trim the work of masked modes when
// the state has none (the flag is refreshed whenever a state is set).
struct TrimScope {   // trimming on for one recording or profiling, off again on every exit
    spk_ctx* c;
    explicit TrimScope(spk_ctx* cc) : c(cc) { c->trim_now = c->defer && c->d_keep; }
    ~TrimScope() { c->trim_now = false; }
};
static void record_step(spk_ctx* c, int parity) {
    TrimScope ts(c);
    record_step_body(c, parity);
}
static void record_step_body(spk_ctx* c, int parity, bool rk_only) {
    const spk_params_t& p = c->p;
    const bool sts = p.supertimestepping && c->nsts > 0 && !rk_only;
    const bool sts_before = sts && !p.sts_every_step && parity == 1;
    const bool sts_after = sts && (p.sts_every_step || parity == 0);
    const bool euler = p.integrator == SPK_INT_EULER;
    const int nst = euler ? 1 : 3;
    if (p.heat_equation) {
        if (!rk_only) {
            DtArgs d = dt_args(c, true);
            k_dt<<<c->nb, 32, 0, c->stream>>>(d, c->sc);
            c->launches++;
        }
        if (sts_before) record_rkl_cycle(c);
        for (int s = 0; s < nst; s++) {
            XfArgs x = xf_args(c, c->U, euler ? XM_EULER : s, false);
            k_heat<<<ew_blocks(c->nc * c->nb), 256, 0, c->stream>>>(x);
            c->launches++;
        }
        if (sts_after) record_rkl_cycle(c);
        return;
    }
    const bool shear = p.shearing != 0;
    if (!rk_only) {
        if (shear) {
            // CleanFieldDivergence at the start of the step (supervisor.cu:184),
            // with the wavevector of the possibly remapped state: with the
            // shearing box it is not fused into the previous step's last stage
            launch_clean(c);
            c->launches += p.mhd ? 2 : 1;
        }
        k_reset_max<<<c->nb, 32, 0, c->stream>>>(c->sc);
        c->launches++;
    }
    // shearing box: stage s uses the wavevector at tremap + csh[s] dt
    // (hydro_mhd_advance.cu:129-131, 148-150)
    const double csh[3] = {0.0, 8.0 / 15.0, 8.0 / 15.0 + -17.0 / 60.0 + 5.0 / 12.0};
    for (int s = 0; s < nst; s++) {
        const bool first = s == 0 && !rk_only;
        c->stage_csh = (shear && !euler) ? csh[s] : 0.0;
        pass_x_inverse(c, c->U, true, euler ? 0 : s);
        pass_y_inverse(c, true);
        if (first) {
            if (sts_before) {
                pass_z_inverse_only(c, true, c->sts_aniso);
                DtArgs d = dt_args(c, true);
                k_dt<<<c->nb, 32, 0, c->stream>>>(d, c->sc);
                c->launches++;
                record_rkl_cycle(c);
                pass_z_products(c, false);
            } else {
                pass_z_products(c, true);
                DtArgs d = dt_args(c, true);
                k_dt<<<c->nb, 32, 0, c->stream>>>(d, c->sc);
                c->launches++;
            }
        } else {
            pass_z_products(c, false);
        }
        pass_y_forward(c, c->nout, c->bufA, c->bufB);
        // the last stage cleans the new u and B: CleanFieldDivergence of the next step
        XfArgs x = xf_args(c, c->U, euler ? XM_EULER : s, s == nst - 1 && !rk_only && !shear);
        xfwd(c, x);
    }
    c->stage_csh = 0.0;
    if (shear) {
        // the remap clock, then RemapAllFields when it passed half a period
        k_shear_end<<<1, 32, 0, c->stream>>>(c->sc, p.lx, p.ly, p.shear);
        const long items = (long)c->F * c->ny * ((c->nzh + SPK_REMAP_KC - 1) / SPK_REMAP_KC);
        const int grid = (int)std::min<long>(items, (long)c->num_sms * 8);
        k_remap<<<grid, 256, sizeof(double2) * (size_t)c->nx * SPK_REMAP_KC, c->stream>>>(c->g, c->U, c->F, c->sc);
        c->launches += 2;
    }
    if (sts_after) {
        if (c->sts_aniso) record_breal(c);
        record_rkl_cycle(c);
    }
}

// TimeStepping::ShiftTime (src/timestepping/shearing_remapping.cu:15-25):
// the remap clock of time t
static double shift_time(const spk_params_t& p, double t) {
    const double h = p.ly / (2.0 * p.shear * p.lx);
    return fmod(t + h, p.ly / (p.shear * p.lx)) - h;
}

// ---------------------------------------------------------------------------
// context creation
// ---------------------------------------------------------------------------
extern "C" void spk_params_default(spk_params_t* p) {
    memset(p, 0, sizeof(*p));
    p->nx = p->ny = p->nz = 32;
    p->lx = p->ly = p->lz = 1.0;
    p->strat_direction = 2;
    p->sts_algorithm = SPK_STS_RKL2;
    p->antialiasing = 1;
    p->nu = p->nu_m = p->nu_th = 1.0;
    p->reynolds_ani = 1.0;
    p->cfl = 1.5; p->cfl_par = 1.0; p->cfl_sts = 1.0; p->safety_source = 0.2;
    p->safety_sts = 1;
    p->t_initial = 0.0; p->t_final = 1.0; p->toutput_flow = 1.0;
    p->integrator = SPK_INT_RK3;
    p->form = SPK_FORM_PLAIN;
    p->closure = 0;
}

static int check_params(const spk_params_t* p, std::string& why) {
    // Parameters::checkParameters (parameters.cu:511-566)
    if (p->incompressible && p->heat_equation) { why = "incompressible and heat_equation modules are mutually exclusive"; return SPK_ERR_CONFIG; }
    if (!p->incompressible && !p->heat_equation) { why = "choose either the incompressible or the heat_equation module"; return SPK_ERR_CONFIG; }
    if (p->boussinesq && !p->incompressible) { why = "Boussinesq requires incompressible module"; return SPK_ERR_CONFIG; }
    if (p->stratification && !p->boussinesq) { why = "stratification requires Boussinesq module"; return SPK_ERR_CONFIG; }
    if (p->mhd && !p->incompressible) { why = "mhd requires incompressible module"; return SPK_ERR_CONFIG; }
    if (p->anisotropic_diffusion && !(p->mhd && p->boussinesq)) { why = "anisotropic_diffusion requires mhd and boussinesq module"; return SPK_ERR_CONFIG; }
    if (p->nx < 2 || p->ny < 2 || p->nz < 2) { why = "grid sizes must be >= 2"; return SPK_ERR_ARG; }
    if (p->nz % 2) { why = "NZ must be even"; return SPK_ERR_UNSUPPORTED; }
    if (p->nx > 1024 || p->ny > 1024 || p->nz > 1024) { why = "axis lengths above 1024 are not supported"; return SPK_ERR_UNSUPPORTED; }
    if (p->supertimestepping && p->sts_algorithm != SPK_STS_STS && p->sts_algorithm != SPK_STS_RKL1 && p->sts_algorithm != SPK_STS_RKL2) {
        why = "sts_algorithm must be sts, rkl1 or rkl2"; return SPK_ERR_CONFIG;
    }
    if (p->form != SPK_FORM_PLAIN && p->form != SPK_FORM_FP32) { why = "unknown form"; return SPK_ERR_ARG; }
    if (p->strat_direction < 0 || p->strat_direction > 2) { why = "strat_direction must be 0, 1 or 2"; return SPK_ERR_ARG; }
    if (p->closure < 0 || p->closure > 3) {
        why = "closure must be 0, 1 (full-field model), 2 (small-scale model) or 3 (tensor network)";
        return SPK_ERR_ARG;
    }
    if (!(p->closure_kc_frac >= 0.0 && p->closure_kc_frac < 1.0)) { why = "closure_kc_frac must be in [0, 1)"; return SPK_ERR_ARG; }
    if (p->closure && (!p->incompressible || p->boussinesq)) { why = "the learned closure covers the HD and MHD modules"; return SPK_ERR_UNSUPPORTED; }
    if (p->closure && p->supertimestepping) { why = "the learned closure with super-time-stepping is not supported"; return SPK_ERR_UNSUPPORTED; }
    if (p->shearing) {
        if (!p->incompressible) { why = "the shearing box needs the incompressible module"; return SPK_ERR_UNSUPPORTED; }
        if (!(p->shear != 0.0) || !std::isfinite(p->shear)) { why = "shearing needs a finite, nonzero shear"; return SPK_ERR_ARG; }
        if (p->closure) { why = "the shearing box with the learned closure is not supported"; return SPK_ERR_UNSUPPORTED; }
    }
    return SPK_OK;
}

// Parameters::Parameters (src/parameters/parameters.cu:59-505) for the keys
// of this path, from a parsed libconfig-format file: every lookup that
// fails (absent, or of another type) keeps the default, as in the reference.
static int params_from_config(const spkcfg::Setting& root, spk_params_t* p) {
    using namespace spkcfg;
    spk_params_default(p);
    get_bool(root, "modules.with2d", &p->with2d);
    get_bool(root, "modules.incompressible", &p->incompressible);
    get_bool(root, "modules.heat_equation", &p->heat_equation);
    get_bool(root, "modules.boussinesq", &p->boussinesq);
    get_bool(root, "modules.stratification", &p->stratification);
    get_int(root, "modules.strat_direction", &p->strat_direction);
    get_bool(root, "modules.mhd", &p->mhd);
    get_bool(root, "modules.anisotropic_diffusion", &p->anisotropic_diffusion);
    get_bool(root, "modules.supertimestepping", &p->supertimestepping);
    get_bool(root, "modules.shearing", &p->shearing);
    get_bool(root, "modules.rotating", &p->rotating);
    // sts_algorithm / sts_variables (:111-156): read only with supertimestepping;
    // no (or an empty) variable list switches it off
    std::vector<std::string> sts_vars;
    if (p->supertimestepping) {
        std::string alg;
        if (get_string(root, "modules.sts_algorithm", &alg)) {
            p->sts_algorithm = alg == "rkl2" ? SPK_STS_RKL2 : (alg == "rkl1" ? SPK_STS_RKL1 : (alg == "sts" ? SPK_STS_STS : 0));
            const Setting* sv = lookup(root, "modules.sts_variables");
            if (sv && (sv->type == T_LIST || sv->type == T_ARRAY) && !sv->items.empty()) {
                for (const Setting& e : sv->items)
                    if (e.type == T_STRING) sts_vars.push_back(e.sval);
            } else {
                p->supertimestepping = 0;
            }
        }
    }
    get_float(root, "physics.boxsize.[0]", &p->lx);
    get_float(root, "physics.boxsize.[1]", &p->ly);
    get_float(root, "physics.boxsize.[2]", &p->lz);
    get_int(root, "physics.gridsize.[0]", &p->nx);
    get_int(root, "physics.gridsize.[1]", &p->ny);
    get_int(root, "physics.gridsize.[2]", &p->nz);
    double re = 1.0, rem = 1.0, reth = 1.0;
    get_float(root, "physics.reynolds", &re);
    get_float(root, "physics.reynolds_magnetic", &rem);
    get_float(root, "physics.reynolds_thermic", &reth);
    p->nu = 1. / re;
    p->nu_m = 1. / rem;
    p->nu_th = 1. / reth;
    get_float(root, "physics.reynolds_anisotropic", &p->reynolds_ani);
    get_float(root, "physics.brunt_vaissala_squared", &p->N2);
    get_float(root, "physics.mti_frequency_squared", &p->OmegaT2);
    get_float(root, "physics.omega", &p->omega);
    get_float(root, "physics.shear", &p->shear);
    get_float(root, "code.cfl", &p->cfl);
    get_float(root, "code.cfl_par", &p->cfl_par);
    get_float(root, "code.cfl_sts", &p->cfl_sts);
    get_int(root, "code.safety_sts", &p->safety_sts);
    get_float(root, "code.safety_source", &p->safety_source);
    get_float(root, "code.t_initial", &p->t_initial);
    get_float(root, "code.t_final", &p->t_final);
    get_bool(root, "code.antialiasing", &p->antialiasing);
    get_float(root, "output.snapshot_step", &p->toutput_flow);
    // STS variables -> bits of the field order of Parameters::popVariablesGrid (:617-638)
    std::vector<std::string> names;
    if (p->heat_equation) names = {"th"};
    else if (p->incompressible) {
        names = {"vx", "vy", "vz"};
        if (p->mhd) { names.push_back("bx"); names.push_back("by"); names.push_back("bz"); }
        if (p->boussinesq) names.push_back("th");
    }
    p->sts_vars_mask = 0;
    for (const std::string& v : sts_vars)
        for (size_t f = 0; f < names.size(); f++)
            if (names[f] == v) p->sts_vars_mask |= 1u << f;
    // with shearing, snapshots only where the box is exactly periodic
    // (parameters.cu:551-562, its arithmetic kept: a step above one period
    // becomes the whole number of periods it holds, not their length)
    if (p->shearing) {
        const double tperiodic = p->ly / (p->shear * p->lx);
        if (p->toutput_flow < tperiodic) p->toutput_flow = tperiodic;
        else p->toutput_flow = (double)(int)(p->toutput_flow / tperiodic);
    }
    std::string why;
    const int rc = check_params(p, why);
    if (rc == SPK_ERR_CONFIG) return fail(nullptr, rc, why);
    return SPK_OK;
}

// Any key of a configuration text, with libconfig's typed lookups (the
// keys of Parameters::Parameters that spk_params_t does not carry: output,
// initial conditions, shearing, ...).  1: found with that type; 0: absent or
// of another type; -1: the text does not parse (spk_last_error(NULL)).
static int cfg_root(const char* text, spkcfg::Setting* root) {
    if (!text) { fail(nullptr, SPK_ERR_ARG, "null configuration text"); return -1; }
    const std::string t(text);
    std::string err;
    if (!spkcfg::Parser(t).parse(*root, err)) { fail(nullptr, SPK_ERR_ARG, "configuration: " + err); return -1; }
    return 0;
}
extern "C" int spk_cfg_lookup_int(const char* text, const char* path, int* out) {
    spkcfg::Setting r;
    if (cfg_root(text, &r) || !path || !out) return -1;
    return spkcfg::get_int(r, path, out) ? 1 : 0;
}
extern "C" int spk_cfg_lookup_bool(const char* text, const char* path, int* out) {
    spkcfg::Setting r;
    if (cfg_root(text, &r) || !path || !out) return -1;
    return spkcfg::get_bool(r, path, out) ? 1 : 0;
}
extern "C" int spk_cfg_lookup_float(const char* text, const char* path, double* out) {
    spkcfg::Setting r;
    if (cfg_root(text, &r) || !path || !out) return -1;
    return spkcfg::get_float(r, path, out) ? 1 : 0;
}
extern "C" int spk_cfg_lookup_string(const char* text, const char* path, char* buf, size_t len) {
    spkcfg::Setting r;
    if (cfg_root(text, &r) || !path || !buf || len == 0) return -1;
    std::string v;
    if (!spkcfg::get_string(r, path, &v)) return 0;
    if (v.size() + 1 > len) { fail(nullptr, SPK_ERR_ARG, std::string("string value of ") + path + " is too long"); return -1; }
    memcpy(buf, v.c_str(), v.size() + 1);
    return 1;
}
extern "C" int spk_cfg_setting_length(const char* text, const char* path) {
    spkcfg::Setting r;
    if (cfg_root(text, &r) || !path) return -1;
    const spkcfg::Setting* st = spkcfg::lookup(r, path);
    if (!st) return -1;
    return (st->type == spkcfg::T_GROUP || st->type == spkcfg::T_ARRAY || st->type == spkcfg::T_LIST) ? (int)st->items.size() : 0;
}

extern "C" int spk_params_from_string(const char* text, spk_params_t* p) {
    if (!text || !p) return fail(nullptr, SPK_ERR_ARG, "null argument");
    const std::string t(text);
    spkcfg::Setting root;
    std::string err;
    if (!spkcfg::Parser(t).parse(root, err)) return fail(nullptr, SPK_ERR_ARG, "configuration: " + err);
    return params_from_config(root, p);
}

extern "C" int spk_params_from_file(const char* path, spk_params_t* p) {
    if (!path || !p) return fail(nullptr, SPK_ERR_ARG, "null argument");
    FILE* fp = fopen(path, "rb");
    if (!fp) return fail(nullptr, SPK_ERR_ARG, std::string("cannot open configuration file ") + path);
    std::string t;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), fp)) > 0) t.append(buf, n);
    fclose(fp);
    spkcfg::Setting root;
    std::string err;
    if (!spkcfg::Parser(t).parse(root, err)) return fail(nullptr, SPK_ERR_ARG, std::string(path) + ": " + err);
    return params_from_config(root, p);
}

static int ctx_init(spk_ctx* c, const spk_params_t* pin, void* stream) {
    c->p = *pin;
    const spk_params_t& p = c->p;
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    if (!c->stream) {
        // graph capture needs a non-legacy stream: create one
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
            return fail(nullptr, SPK_ERR_CUDA, "cudaStreamCreateWithFlags failed");
        c->own_stream = true;
    }
    c->fp32 = p.form == SPK_FORM_FP32;
    // Parameters::popVariablesGrid (parameters.cu:568-654)
    c->F = 0; c->VX = c->VY = c->VZ = c->BX = c->BY = c->BZ = c->TH = c->VEL = c->MAG = 0;
    if (p.heat_equation) { c->TH = 0; c->F = 1; }
    else {
        c->VX = 0; c->VY = 1; c->VZ = 2; c->F = 3;
        if (p.mhd) { c->BX = 3; c->BY = 4; c->BZ = 5; c->MAG = 3; c->F += 3; if (p.boussinesq) { c->TH = 6; c->F += 1; } }
        else if (p.boussinesq) { c->TH = 3; c->F += 1; }
    }
    c->nx = p.nx; c->ny = p.ny; c->nz = p.nz; c->nzh = p.nz / 2 + 1;
    c->nc = (size_t)c->nx * c->ny * c->nzh;
    c->nr = (size_t)c->nx * c->ny * c->nz;
    // Wavevector::Wavevector (wavevector.cu:50-112): host FP64, exact expressions
    c->kx.resize(c->nx); c->ky.resize(c->ny); c->kz.resize(c->nzh);
    c->mx.assign(c->nx, 1.0); c->my.assign(c->ny, 1.0); c->mz.assign(c->nzh, 1.0);
    volatile double twopi = 2.0 * M_PI;
    for (int i = 0; i < c->nx; i++) c->kx[i] = twopi / p.lx * (fmod((double)i + ((double)c->nx / 2), c->nx) - (double)c->nx / 2);
    for (int j = 0; j < c->ny; j++) c->ky[j] = twopi / p.ly * (fmod((double)j + ((double)c->ny / 2), c->ny) - (double)c->ny / 2);
    for (int k = 0; k < c->nzh; k++) c->kz[k] = p.with2d ? 0.0 : twopi / p.lz * (double)k;
    c->kxmax = 2.0 * M_PI / p.lx * ((c->nx / 2) - 1);
    c->kymax = 2.0 * M_PI / p.ly * ((c->ny / 2) - 1);
    c->kzmax = 2.0 * M_PI / p.lz * ((c->nz / 2) - 1);
    if (p.with2d) c->kzmax = 0.0;
    if (p.antialiasing) {
        volatile double two3 = 2.0 / 3.0;
        const double tx = two3 * c->kxmax, ty = two3 * c->kymax, tz = two3 * c->kzmax;
        for (int i = 0; i < c->nx; i++) if (fabs(c->kx[i]) > tx) c->mx[i] = 0.0;
        for (int j = 0; j < c->ny; j++) if (fabs(c->ky[j]) > ty) c->my[j] = 0.0;
        for (int k = 0; k < c->nzh; k++) if (fabs(c->kz[k]) > tz) c->mz[k] = 0.0;
        c->kxmax = (2.0 / 3.0) * c->kxmax;
        c->kymax = (2.0 / 3.0) * c->kymax;
        c->kzmax = (2.0 / 3.0) * c->kzmax;
    }
    c->kmax = pow(c->kxmax * c->kxmax + c->kymax * c->kymax + c->kzmax * c->kzmax, 0.5);
    c->kz_keep = 0;
    while (c->kz_keep < c->nzh && c->mz[c->kz_keep] != 0.0) c->kz_keep++;
    for (int k = c->kz_keep; k < c->nzh; k++)
        if (c->mz[k] != 0.0) return fail(nullptr, SPK_ERR_UNSUPPORTED, "kz mask is not a prefix");

    // STS variables (RKLegendre ctor, rkl.cu:40-58)
    c->sts_mask = 0; c->nsts = 0; c->sts_aniso = c->sts_iso = false;
    if (p.supertimestepping) {
        for (int f = 0; f < c->F; f++) {
            if ((p.sts_vars_mask >> f) & 1u) {
                c->sts_mask |= 1u << f;
                int kind;
                if (p.heat_equation || (p.boussinesq && f == c->TH)) kind = (p.anisotropic_diffusion ? 3 : 2);
                else if (p.mhd && f >= c->MAG && f < c->MAG + 3) kind = 1;
                else kind = 0;
                c->sts_fields[c->nsts] = f;
                c->sts_kind[c->nsts] = kind;
                c->nsts++;
                if (kind == 3) c->sts_aniso = true; else c->sts_iso = true;
            }
        }
        if (c->sts_aniso && p.mhd && (c->sts_mask >> c->MAG & 7u))
            return fail(nullptr, SPK_ERR_UNSUPPORTED, "super-time-stepping of B together with anisotropic conduction is not supported");
    }
    c->aniso_rhs = p.anisotropic_diffusion && p.boussinesq && !((c->sts_mask >> c->TH) & 1u);
    // bound on the stage count of one super-time-stepping cycle (the graph
    // records this many stages; k_dt flags a cycle that needs more)
    c->rkl_smax = 0;
    if (c->nsts > 0) {
        double r;
        if (p.heat_equation) {
            const double gam = (c->kxmax * c->kxmax + c->kymax * c->kymax + c->kzmax * c->kzmax) * p.nu_th;
            const double dts = p.cfl_par / gam;
            double dtm = p.fixed_dt > 0.0 ? p.fixed_dt : p.t_final - p.t_initial;
            r = std::max(1.0, dtm / dts);
        } else {
            r = std::max(1.0, (double)p.safety_sts);
        }
        int s = sts_stage_count(p.sts_algorithm, r);
        if (s < 1) s = SPK_RKL_MAX;   // no STS root: take the cap
        c->rkl_smax = std::min(SPK_RKL_MAX - 1, 1 + s);
    }

    // channel layout of the main pipeline
    int ch = 0;
    c->ch_u = c->ch_b = c->ch_th = c->ch_gx = c->ch_gy = -1;
    if (p.incompressible) { c->ch_u = ch; ch += 3; }
    if (p.mhd) { c->ch_b = ch; ch += 3; }
    if (p.boussinesq) { c->ch_th = ch; ch += 1; }
    c->nin_base = ch;
    if (c->aniso_rhs) { c->ch_gx = ch; c->ch_gy = ch + 1; ch += 2; }
    c->ch_dx = c->ch_dy = -1;
    c->ncl_half = 0;
    if (p.closure == 1 || p.closure == 3) {
        c->ncl_half = p.mhd ? 6 : 3;
        c->ch_dx = ch; ch += c->ncl_half;
        c->ch_dy = ch; ch += c->ncl_half;
    } else if (p.closure == 2) {
        // every gradient component from the x inverse, of the small scales only
        c->ngrad = p.mhd ? 18 : 9;
        c->ch_dx = ch; ch += c->ngrad;
        const double kc = std::min(c->kxmax, std::min(c->kymax, c->kzmax));
        const double f = p.closure_kc_frac > 0.0 ? p.closure_kc_frac : 0.5;
        c->hp_k2 = f * f * kc * kc;
    }
    c->delta2 = pow(M_PI / c->kxmax * M_PI / c->kymax * M_PI / c->kzmax, 2.0 / 3.0);
    c->nin = ch;
    c->nkx = c->nky = 0;
    for (int i = 0; i < c->nx; i++) c->nkx += c->mx[i] != 0.0;
    for (int j = 0; j < c->ny; j++) c->nky += c->my[j] != 0.0;
    {
        // Wavevector: deltak = 2 pi / min(l), nbins = (int)(kmax/deltak + 0.5) (wavevector.cu:100-111)
        double lmin = p.lx;
        if (p.ly < lmin) lmin = p.ly;
        if (p.lz < lmin) lmin = p.lz;
        c->deltak = 2.0 * M_PI / lmin;
        c->nbins = (int)(c->kmax / c->deltak + 0.5);
    }
    // (the shearing box's source terms and sheared projection act on masked
    // modes too: no deferral)
    c->defer = p.incompressible && !p.boussinesq && c->sts_mask == 0 && p.integrator == SPK_INT_RK3 &&
               c->nkx > 0 && c->nky > 0 && c->kz_keep > 0 && !p.shearing;
    int oc = 0;
    c->out_T = c->out_E = c->out_F = c->out_Q = -1;
    if (p.incompressible) { c->out_T = oc; oc += 5; }
    if (p.mhd) { c->out_E = oc; oc += 3; }
    if (p.boussinesq) { c->out_F = oc; oc += 3; }
    if (c->aniso_rhs) { c->out_Q = oc; oc += 3; }
    c->nout = oc;
    c->nbuf_ch = std::max(std::max(c->nin + 1, c->nout), 3);

    // transform lengths the register-resident FFT covers
    if (!regfft_length_ok(c->nx) || !regfft_length_ok(c->ny) || !regfft_length_ok(c->nz))
        return fail(nullptr, SPK_ERR_UNSUPPORTED, "axis lengths must be 2^k (2..1024) or 3*2^k (6..768)");
    c->plan_x.n = c->nx;
    c->plan_y.n = c->ny;
    c->plan_z.n = c->nz;
    return SPK_OK;
}

static int ctx_alloc(spk_ctx* c) {
    const size_t nc = c->nc;
    const size_t cs = csize(c);
    // device properties and the tensor-map encoder (driver entry point,
    // resolved through the runtime: no link-time dependency on libcuda)
    {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
        if (!g_encode) {
            cudaDriverEntryPointQueryResult q;
            void* fn = nullptr;
            CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
            if (q != cudaDriverEntryPointSuccess || !fn) return fail(c, SPK_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
            g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
        }
    }
    // tables
    CK(cudaMalloc(&c->d_tab, sizeof(double) * (2 * ((size_t)c->nx + c->ny + c->nzh))));
    double* t = c->d_tab;
    CK(cudaMemcpy(t, c->kx.data(), sizeof(double) * c->nx, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t + c->nx, c->ky.data(), sizeof(double) * c->ny, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t + c->nx + c->ny, c->kz.data(), sizeof(double) * c->nzh, cudaMemcpyHostToDevice));
    double* m = t + c->nx + c->ny + c->nzh;
    CK(cudaMemcpy(m, c->mx.data(), sizeof(double) * c->nx, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m + c->nx, c->my.data(), sizeof(double) * c->ny, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(m + c->nx + c->ny, c->mz.data(), sizeof(double) * c->nzh, cudaMemcpyHostToDevice));
    c->g.nx = c->nx; c->g.ny = c->ny; c->g.nz = c->nz; c->g.nzh = c->nzh;
    c->g.nzs = pass_row(c->nzh, c->fp32);
    c->g.ncs = (size_t)c->nx * c->ny * c->g.nzs;
    c->g.kz_keep = c->kz_keep; c->g.nc = nc;
    c->g.kx = t; c->g.ky = t + c->nx; c->g.kz = t + c->nx + c->ny;
    c->g.mx = m; c->g.my = m + c->nx; c->g.mz = m + c->nx + c->ny;
    // twiddles
    const size_t ntw = (size_t)c->nx + c->ny + c->nz;
    CK(cudaMalloc(&c->d_tw, cs * ntw));
    std::vector<double> tw;
    size_t off = 0;
    FftPlan* pls[3] = {&c->plan_x, &c->plan_y, &c->plan_z};
    for (int a = 0; a < 3; a++) {
        const int n = pls[a]->n;
        twiddles(n, tw);
        void* dst = (char*)c->d_tw + off * cs;
        if (c->fp32) {
            std::vector<float> tf(tw.begin(), tw.end());
            CK(cudaMemcpy(dst, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(dst, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice));
        }
        pls[a]->tw = dst;
        off += n;
    }
    // state and buffers
    const size_t nb = (size_t)c->nb;
    CK(cudaMalloc(&c->U, sizeof(double2) * nc * c->F * nb));
    CK(cudaMalloc(&c->S, sizeof(double2) * nc * c->F * nb));
    CK(cudaMemset(c->U, 0, sizeof(double2) * nc * c->F * nb));
    CK(cudaMemset(c->S, 0, sizeof(double2) * nc * c->F * nb));
    if (c->p.incompressible) {
        CK(cudaMalloc(&c->bufA, cs * c->g.ncs * c->nbuf_ch * nb));
        CK(cudaMalloc(&c->bufB, cs * c->g.ncs * c->nbuf_ch * nb));
        CK(cudaMemset(c->bufA, 0, cs * c->g.ncs * c->nbuf_ch * nb));
        CK(cudaMemset(c->bufB, 0, cs * c->g.ncs * c->nbuf_ch * nb));
    }
    // stage scratch: RKL2 keeps Uc0, Uc1 and dU0, RKL1 only Uc1, STS none
    if (c->nsts > 0 && c->p.sts_algorithm != SPK_STS_STS) {
        CK(cudaMalloc(&c->Uc1, sizeof(double2) * nc * c->nsts));
        CK(cudaMemset(c->Uc1, 0, sizeof(double2) * nc * c->nsts));
    }
    if (c->nsts > 0 && c->p.sts_algorithm == SPK_STS_RKL2) {
        CK(cudaMalloc(&c->Uc0, sizeof(double2) * nc * c->nsts));
        CK(cudaMalloc(&c->dU0, sizeof(double2) * nc * c->nsts));
        CK(cudaMemset(c->Uc0, 0, sizeof(double2) * nc * c->nsts));
        CK(cudaMemset(c->dU0, 0, sizeof(double2) * nc * c->nsts));
    }
    if (c->sts_aniso) {
        CK(cudaMalloc(&c->rA, cs * c->g.ncs * 3));
        CK(cudaMalloc(&c->rB, cs * c->g.ncs * 3));
        CK(cudaMemset(c->rA, 0, cs * c->g.ncs * 3));
        CK(cudaMemset(c->rB, 0, cs * c->g.ncs * 3));
        CK(cudaMalloc(&c->breal, (c->fp32 ? sizeof(float) : sizeof(double)) * c->nr * 3));
    }
    CK(cudaMalloc(&c->sc, sizeof(DevScalars) * nb));
    CK(cudaMallocHost(&c->h_sc, sizeof(DevScalars) * nb));
    memset(c->h_sc, 0, sizeof(DevScalars) * nb);
    for (size_t b = 0; b < nb; b++) {
        c->h_sc[b].t = c->p.t_initial;
        c->h_sc[b].nu = c->bnu.empty() ? c->p.nu : c->bnu[b];
        c->h_sc[b].nu_m = c->bnu_m.empty() ? c->p.nu_m : c->bnu_m[b];
        c->h_sc[b].nu_th = c->bnu_th.empty() ? c->p.nu_th : c->bnu_th[b];
        c->h_sc[b].masked_live = 1;
        // the main loop starts the remap clock from the time (supervisor.cu:171-175)
        c->h_sc[b].tremap = c->p.shearing ? shift_time(c->p, c->p.t_initial) : 0.0;
    }
    CK(cudaMemcpy(c->sc, c->h_sc, sizeof(DevScalars) * nb, cudaMemcpyHostToDevice));
    c->g.shear = c->p.shearing ? c->p.shear : 0.0;
    c->g.csh = 0.0;
    c->g.shsc = c->sc;
    CK(cudaMalloc(&c->d_sums, sizeof(double) * 16));
    CK(cudaMallocHost(&c->h_sums, sizeof(double) * 16));
    if (c->p.closure) {
        const size_t np = (size_t)spk_closure_nparam(c->p.closure);
        CK(cudaMalloc(&c->d_cparams, sizeof(float) * np));
        CK(cudaMemset(c->d_cparams, 0, sizeof(float) * np));
        if (c->p.closure == 3) {
            CK(cudaMalloc(&c->d_cimg, (size_t)C3_ALL_BYTES));
            CK(cudaMemset(c->d_cimg, 0, (size_t)C3_ALL_BYTES));
        }
    }
    CK(cudaMalloc(&c->d_spec, sizeof(double) * (size_t)(c->nbins + 1)));
    if (c->nkx > 0 && c->nky > 0) {
        // kept x and y indices (deferred masked modes, compact tile walks)
        std::vector<int> keep;
        for (int i = 0; i < c->nx; i++) if (c->mx[i] != 0.0) keep.push_back(i);
        for (int j = 0; j < c->ny; j++) if (c->my[j] != 0.0) keep.push_back(j);
        CK(cudaMalloc(&c->d_keep, sizeof(int) * keep.size()));
        CK(cudaMemcpy(c->d_keep, keep.data(), sizeof(int) * keep.size(), cudaMemcpyHostToDevice));
    }
    return SPK_OK;
}

static void ctx_free(spk_ctx* c) {
    for (int i = 0; i < 2; i++) if (c->have_graph[i]) cudaGraphExecDestroy(c->gexec[i]);
    for (int i = 0; i < 2; i++) if (c->have_fgraph[i]) cudaGraphExecDestroy(c->fgexec[i]);
    cudaFree(c->d_tab); cudaFree(c->d_tw); cudaFree(c->U); cudaFree(c->S);
    cudaFree(c->bufA); cudaFree(c->bufB); cudaFree(c->rA); cudaFree(c->rB); cudaFree(c->breal);
    cudaFree(c->Uc0); cudaFree(c->Uc1); cudaFree(c->dU0); cudaFree(c->sc); cudaFree(c->d_sums);
    cudaFree(c->d_cparams);
    cudaFree(c->d_cimg);
    cudaFree(c->d_keep);
    cudaFree(c->d_spec);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    if (c->h_sums) cudaFreeHost(c->h_sums);
    if (c->own_stream) cudaStreamDestroy(c->stream);
}

static int launch_status(spk_ctx* c) {
    if (c->sticky) return c->sticky;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, SPK_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return SPK_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int spk_ctx_create(const spk_params_t* p, void* stream, spk_ctx** out) {
    if (!p || !out) return fail(nullptr, SPK_ERR_ARG, "null argument");
    *out = nullptr;
    std::string why;
    int rc = check_params(p, why);
    if (rc != SPK_OK) return fail(nullptr, rc, why);
    spk_ctx* c = new spk_ctx();
    memset(c->have_graph, 0, sizeof(c->have_graph));
    c->d_tab = nullptr; c->d_tw = nullptr; c->U = c->S = nullptr; c->bufA = c->bufB = nullptr;
    c->rA = c->rB = c->breal = nullptr; c->Uc0 = c->Uc1 = c->dU0 = nullptr; c->sc = nullptr;
    c->h_sc = nullptr; c->d_sums = nullptr; c->h_sums = nullptr; c->h_step = 0; c->sticky = 0;
    c->launches = 0; c->kernels_per_step[0] = c->kernels_per_step[1] = 0; c->bad_job = false; c->bad_why = ""; c->user_U = nullptr; c->dirty = true;
    rc = ctx_init(c, p, stream);
    if (rc != SPK_OK) { delete c; return rc; }
    rc = ctx_alloc(c);
    if (rc != SPK_OK) {
        g_create_error = c->err;
        ctx_free(c);
        delete c;
        return rc;
    }
    *out = c;
    return SPK_OK;
}

extern "C" int spk_ctx_destroy(spk_ctx* c) {
    if (!c) return SPK_ERR_ARG;
    cudaStreamSynchronize(c->stream);
    ctx_free(c);
    delete c;
    return SPK_OK;
}

extern "C" int spk_sizes(const spk_ctx* c, int* nf, size_t* ncx) {
    if (!c) return SPK_ERR_ARG;
    if (nf) *nf = c->F;
    if (ncx) *ncx = c->nc;
    return SPK_OK;
}

extern "C" int spk_set_state(spk_ctx* c, const double* U, int where) {
    if (!c || !U) return SPK_ERR_ARG;
    CK(cudaMemcpyAsync(c->U, U, sizeof(double2) * c->nc * c->F, where ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream));
    c->dirty = true;
    return SPK_OK;
}

extern "C" int spk_get_state(spk_ctx* c, double* U, int where) {
    if (!c || !U) return SPK_ERR_ARG;
    CK(cudaMemcpyAsync(U, c->U, sizeof(double2) * c->nc * c->F, where ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c->stream));
    if (where) CK(cudaStreamSynchronize(c->stream));
    return SPK_OK;
}

extern "C" int spk_set_time(spk_ctx* c, double t, int step, double t_lastsnap) {
    if (!c) return SPK_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(c->h_sc, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost));
    // a new time restarts the remap clock from it (executeMainLoop's ShiftTime
    // after a restart, supervisor.cu:171-175); the same time keeps the clock
    if (c->p.shearing && t != c->h_sc->t) c->h_sc->tremap = shift_time(c->p, t);
    c->h_sc->t = t; c->h_sc->step = step; c->h_sc->t_lastsnap = t_lastsnap;
    CK(cudaMemcpy(c->sc, c->h_sc, sizeof(DevScalars), cudaMemcpyHostToDevice));
    c->h_step = step;
    return SPK_OK;
}

static int pull_scalars(spk_ctx* c) {
    CK(cudaMemcpyAsync(c->h_sc, c->sc, sizeof(DevScalars) * c->nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SPK_OK;
}

extern "C" int spk_get_time(spk_ctx* c, double* t, double* dt, int* step) {
    if (!c) return SPK_ERR_ARG;
    int rc = pull_scalars(c);
    if (rc) return rc;
    if (t) *t = c->h_sc->t;
    if (dt) *dt = c->h_sc->dt;
    if (step) *step = c->h_sc->step;
    return SPK_OK;
}

static void launch_masked_scan(spk_ctx* c);
static void launch_clean(spk_ctx* c) {
    const size_t bs = (size_t)c->F * c->nc;
    if (c->p.incompressible)
        k_clean<<<ew_blocks(c->nc * c->nb), 256, 0, c->stream>>>(c->g, c->U + (size_t)c->VEL * c->nc, bs, c->nb);
    if (c->p.mhd)
        k_clean<<<ew_blocks(c->nc * c->nb), 256, 0, c->stream>>>(c->g, c->U + (size_t)c->MAG * c->nc, bs, c->nb);
    launch_masked_scan(c);
    c->dirty = false;
}

// The masked-content flag of the deferred modes (DevScalars::masked_live)
// for the current state array.
static void launch_masked_scan(spk_ctx* c) {
    const size_t bs = (size_t)c->F * c->nc;
    if (c->defer && c->d_keep) {
        // is there content outside the 2/3 mask to carry through the steps?
        const dim3 grid((unsigned)std::min<size_t>((c->nc + 255) / 256, (size_t)c->num_sms * 4), (unsigned)c->nb);
        k_masked_scan<<<grid, 256, 0, c->stream>>>(c->g, c->U, c->F, bs, c->sc);
        k_masked_flag<<<c->nb, 32, 0, c->stream>>>(c->sc);
    }
}

extern "C" int spk_clean_divergence(spk_ctx* c) {
    if (!c) return SPK_ERR_ARG;
    launch_clean(c);
    return launch_status(c);
}

extern "C" int spk_compute_dt(spk_ctx* c, double* dt_hyp, double* dt_par, double* dt_sts, double* dt_cur) {
    if (!c) return SPK_ERR_ARG;
    if (c->p.incompressible) {
        k_reset_max<<<1, 32, 0, c->stream>>>(c->sc);
        if (c->closure_on) {
            // the closure's maxima come from the products pass
            pass_x_inverse(c, c->U, true);
            pass_y_inverse(c, true);
            pass_z_products(c, true);
        } else {
            pass_x_inverse(c, c->U, false);
            pass_y_inverse(c, false);
            pass_z_inverse_only(c, true, c->sts_aniso);
        }
    }
    DtArgs d = dt_args(c, false);
    k_dt<<<1, 32, 0, c->stream>>>(d, c->sc);
    int rc = launch_status(c);
    if (rc) return rc;
    rc = pull_scalars(c);
    if (rc) return rc;
    if (dt_hyp) *dt_hyp = c->h_sc->dt_hyp;
    if (dt_par) *dt_par = c->h_sc->dt_par;
    if (dt_sts) *dt_sts = c->h_sc->dt_sts;
    if (dt_cur) *dt_cur = c->h_sc->dt;
    if (c->h_sc->nonfinite) return fail(c, SPK_ERR_NONFINITE, "non-finite value in the real-space fields");
    return SPK_OK;
}

extern "C" int spk_compute_dfield(spk_ctx* c, const double* Uin, double* dUout) {
    if (!c || !Uin || !dUout) return SPK_ERR_ARG;
    double2* U = (double2*)Uin;
    if (c->p.heat_equation) {
        XfArgs x = xf_args(c, U, XM_DFIELD, false);
        x.out = (double2*)dUout;
        k_heat<<<ew_blocks(c->nc), 256, 0, c->stream>>>(x);
        return launch_status(c);
    }
    c->user_U = U;
    pass_x_inverse(c, U, true);
    c->user_U = nullptr;
    pass_y_inverse(c, true);
    pass_z_products(c, false);
    pass_y_forward(c, c->nout, c->bufA, c->bufB);
    XfArgs x = xf_args(c, U, XM_DFIELD, false);
    x.out = (double2*)dUout;
    xfwd(c, x);
    return launch_status(c);
}

// Drops every recorded step graph (the pass layout or schedule changed).
static void drop_graphs(spk_ctx* c) {
    for (int i = 0; i < 2; i++) {
        if (c->have_graph[i]) { cudaGraphExecDestroy(c->gexec[i]); c->have_graph[i] = false; }
        if (c->have_fgraph[i]) { cudaGraphExecDestroy(c->fgexec[i]); c->have_fgraph[i] = false; }
    }
}

// Records one main-loop step of the current state array (c->U) into *ge.
static int capture_step(spk_ctx* c, int par, cudaGraphExec_t* ge) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const long l0 = c->launches;
    record_step(c, par);
    c->kernels_per_step[par] = (int)(c->launches - l0);
    if (c->sticky) {
        cudaGraph_t gbad;
        cudaStreamEndCapture(c->stream, &gbad);
        if (gbad) cudaGraphDestroy(gbad);
        return c->sticky;
    }
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) return fail(c, SPK_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(c, SPK_ERR_CUDA, std::string("graph instantiation: ") + cudaGetErrorString(e));
    return SPK_OK;
}

extern "C" int spk_advance(spk_ctx* c, int nsteps) {
    if (!c || nsteps < 0) return SPK_ERR_ARG;
    const bool alternate = c->p.supertimestepping && c->nsts > 0 && !c->p.sts_every_step;
    // Each step ends with the divergence cleaning of the next step fused into
    // its last update; a state set from outside is cleaned here once.
    if (nsteps > 0 && c->dirty) {
        launch_clean(c);
        int rc = launch_status(c);
        if (rc) return rc;
    }
    for (int it = 0; it < nsteps; it++) {
        const int par = alternate ? (c->h_step & 1) : 0;
        if (!c->have_graph[par]) {
            int rc = capture_step(c, par, &c->gexec[par]);
            if (rc) return rc;
            c->have_graph[par] = true;
        }
        CK(cudaGraphLaunch(c->gexec[par], c->stream));
        c->h_step++;
    }
    return SPK_OK;
}

// ---------------------------------------------------------------------------
// Entry points on the caller's state array (the reference's d_all_fields)
// ---------------------------------------------------------------------------
// For one call the caller's array takes the place of the context's state.
// Afterwards the context's own state is marked as set from outside, so that
// its next step re-derives the masked-content flag the call overwrote.
struct StateSwap {
    spk_ctx* c;
    double2* saved;
    StateSwap(spk_ctx* cc, double2* U) : c(cc), saved(cc->U) { c->U = U; }
    ~StateSwap() { c->U = saved; c->dirty = true; }
};

extern "C" int spk_advance_fields(spk_ctx* c, double* Uin, int nsteps) {
    if (!c || !Uin || nsteps < 0) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_advance_fields acts on single-box contexts");
    if (nsteps == 0) return SPK_OK;
    double2* U = (double2*)Uin;
    const bool alternate = c->p.supertimestepping && c->nsts > 0 && !c->p.sts_every_step;
    StateSwap sw(c, U);
    // the caller may have changed the array since the last call: clean it, as
    // each iteration of the reference's main loop does
    launch_clean(c);
    int rc = launch_status(c);
    if (rc) return rc;
    if (c->fields_graph_ptr != U) {
        for (int i = 0; i < 2; i++)
            if (c->have_fgraph[i]) { cudaGraphExecDestroy(c->fgexec[i]); c->have_fgraph[i] = false; }
        c->fields_graph_ptr = U;
    }
    for (int it = 0; it < nsteps; it++) {
        const int par = alternate ? (c->h_step & 1) : 0;
        if (!c->have_fgraph[par]) {
            rc = capture_step(c, par, &c->fgexec[par]);
            if (rc) return rc;
            c->have_fgraph[par] = true;
        }
        CK(cudaGraphLaunch(c->fgexec[par], c->stream));
        c->h_step++;
    }
    return SPK_OK;
}

extern "C" int spk_rk3_fields(spk_ctx* c, double* Uin) {
    if (!c || !Uin) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_rk3_fields acts on single-box contexts");
    StateSwap sw(c, (double2*)Uin);
    launch_masked_scan(c);
    record_step_body(c, 0, true);
    return launch_status(c);
}

extern "C" int spk_compute_dt_fields(spk_ctx* c, const double* Uin, double* dt_hyp, double* dt_par, double* dt_sts,
                                     double* dt_cur) {
    if (!c || !Uin) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_compute_dt_fields acts on single-box contexts");
    StateSwap sw(c, (double2*)Uin);
    return spk_compute_dt(c, dt_hyp, dt_par, dt_sts, dt_cur);
}

extern "C" int spk_rkl_cycle_fields(spk_ctx* c, double* Uin, int* s_out) {
    if (!c || !Uin) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_rkl_cycle_fields acts on single-box contexts");
    StateSwap sw(c, (double2*)Uin);
    return spk_rkl_cycle(c, s_out);
}

extern "C" int spk_rkl_cycle(spk_ctx* c, int* s_out) {
    if (!c) return SPK_ERR_ARG;
    if (c->nsts == 0) { if (s_out) *s_out = 0; return SPK_OK; }
    record_rkl_cycle(c);
    int rc = launch_status(c);
    if (rc) return rc;
    rc = pull_scalars(c);
    if (rc) return rc;
    if (s_out) *s_out = c->h_sc->s_rkl;
    return SPK_OK;
}

extern "C" int spk_to_real(spk_ctx* c, double* R) {
    if (!c || !R) return SPK_ERR_ARG;
    if (!c->p.incompressible) {
        // heat equation: transform the single field through a temporary pipeline
        return fail(c, SPK_ERR_UNSUPPORTED, "spk_to_real needs the incompressible module");
    }
    pass_x_inverse(c, c->U, false);
    pass_y_inverse(c, false);
    ZArgs z = z_args(c);
    z.mode = ZM_TO_REAL;
    set_inputs(c, z, false);
    z.real_out = R;
    zpass(c, z);
    return launch_status(c);
}

extern "C" int spk_synchronize(spk_ctx* c) {
    if (!c) return SPK_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    int rc = pull_scalars(c);
    if (rc) return rc;
    for (int b = 0; b < c->nb; b++) {
        const std::string box = c->nb > 1 ? " (box " + std::to_string(b) + " of the group)" : "";
        if (c->h_sc[b].err == 1) return fail(c, SPK_ERR_ARG, "super-time-stepping stage count exceeded the recorded bound" + box);
        if (c->h_sc[b].err == 2) return fail(c, SPK_ERR_CUDA, "a bulk/TMA copy wait ran out in a pass kernel" + box);
        if (c->h_sc[b].nonfinite) return fail(c, SPK_ERR_NONFINITE, "non-finite value in the real-space fields" + box);
    }
    return SPK_OK;
}

// Energy budgets of box b (0 for a single-box context).
static int box_budgets(spk_ctx* c, int b, spk_budgets_t* out) {
    CK(cudaMemsetAsync(c->d_sums, 0, sizeof(double) * 16, c->stream));
    if (c->nc >= (1ull << 31)) return fail(c, SPK_ERR_UNSUPPORTED, "budgets: more than 2^31 modes per box");
    k_budgets<<<ew_blocks(c->nc), 256, 0, c->stream>>>(c->g, c->U + (size_t)b * c->F * c->nc, c->F, c->d_sums,
                                                         FastDiv::make((unsigned)c->nzh), FastDiv::make((unsigned)c->ny));
    CK(cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(double) * 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double n2 = (double)c->nr * (double)c->nr;
    memset(out, 0, sizeof(*out));
    for (int f = 0; f < c->F && f < 8; f++) {
        out->energy[f] = 0.5 * c->h_sums[2 * f] / n2;
        out->dissipation[f] = c->h_sums[2 * f + 1] / n2;
    }
    return SPK_OK;
}

extern "C" int spk_budgets(spk_ctx* c, spk_budgets_t* out) {
    if (!c || !out) return SPK_ERR_ARG;
    return box_budgets(c, 0, out);
}

// ---------------------------------------------------------------------------
// Ensembles of independent boxes.  The reference runs one box per process.
// Here boxes that share everything but their viscosities (nu, nu_m, nu_th)
// form a group: one context whose arrays hold the group's boxes side by
// side, whose pass kernels cover all of them in one launch (the box is part
// of the tile / line / mode index) and whose DevScalars hold one dt and one
// set of viscosities per box.  Groups run as parallel branches of one CUDA
// graph, so an ensemble step is a single graph launch of a few launches per
// group.
// ---------------------------------------------------------------------------
static bool same_group(const spk_params_t& a, const spk_params_t& b) {
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.lx == b.lx && a.ly == b.ly && a.lz == b.lz &&
           a.incompressible == b.incompressible && a.heat_equation == b.heat_equation && a.mhd == b.mhd &&
           a.boussinesq == b.boussinesq && a.stratification == b.stratification &&
           a.strat_direction == b.strat_direction && a.anisotropic_diffusion == b.anisotropic_diffusion &&
           a.supertimestepping == b.supertimestepping && a.sts_algorithm == b.sts_algorithm &&
           a.sts_vars_mask == b.sts_vars_mask && a.with2d == b.with2d && a.antialiasing == b.antialiasing &&
           a.reynolds_ani == b.reynolds_ani && a.N2 == b.N2 && a.OmegaT2 == b.OmegaT2 && a.cfl == b.cfl &&
           a.cfl_par == b.cfl_par && a.cfl_sts == b.cfl_sts && a.safety_source == b.safety_source &&
           a.safety_sts == b.safety_sts && a.t_initial == b.t_initial && a.t_final == b.t_final &&
           a.toutput_flow == b.toutput_flow && a.fixed_dt == b.fixed_dt && a.integrator == b.integrator &&
           a.sts_every_step == b.sts_every_step && a.form == b.form && a.closure == b.closure;
}

// A context for nb boxes of one geometry (nu, nu_m, nu_th per box).
static int ctx_create_group(const spk_params_t& p0, const std::vector<double>& nu, const std::vector<double>& nu_m,
                            const std::vector<double>& nu_th, spk_ctx** out) {
    std::string why;
    int rc = check_params(&p0, why);
    if (rc != SPK_OK) return fail(nullptr, rc, why);
    spk_ctx* c = new spk_ctx();
    memset(c->have_graph, 0, sizeof(c->have_graph));
    c->d_tab = nullptr; c->d_tw = nullptr; c->U = c->S = nullptr; c->bufA = c->bufB = nullptr;
    c->rA = c->rB = c->breal = nullptr; c->Uc0 = c->Uc1 = c->dU0 = nullptr; c->sc = nullptr;
    c->h_sc = nullptr; c->d_sums = nullptr; c->h_sums = nullptr; c->h_step = 0; c->sticky = 0;
    c->launches = 0; c->kernels_per_step[0] = c->kernels_per_step[1] = 0; c->bad_job = false; c->bad_why = "";
    c->user_U = nullptr; c->dirty = true;
    c->nb = (int)nu.size();
    c->bnu = nu; c->bnu_m = nu_m; c->bnu_th = nu_th;
    rc = ctx_init(c, &p0, nullptr);
    if (rc != SPK_OK) { delete c; return rc; }
    if (c->nsts > 0 && c->nb > 1) {
        ctx_free(c);
        delete c;
        return fail(nullptr, SPK_ERR_UNSUPPORTED, "super-time-stepping boxes cannot share a group");
    }
    if ((size_t)c->nb * c->nc >= (1ull << 31)) {
        ctx_free(c);
        delete c;
        return fail(nullptr, SPK_ERR_UNSUPPORTED, "a group of boxes above 2^31 modes");
    }
    rc = ctx_alloc(c);
    if (rc != SPK_OK) {
        g_create_error = c->err;
        ctx_free(c);
        delete c;
        return rc;
    }
    *out = c;
    return SPK_OK;
}

struct spk_ensemble {
    std::vector<spk_ctx*> group;               // one context per geometry
    std::vector<std::pair<int, int>> where;    // box -> (group, index in the group)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;             // one per group
    cudaGraphExec_t gexec = nullptr;
    bool have_graph = false;
    int kernels_per_step = 0;
};

static int ens_fail(const std::string& msg, int code) { return fail(nullptr, code, msg); }

extern "C" int spk_ensemble_destroy(spk_ensemble* e) {
    if (!e) return SPK_ERR_ARG;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->have_graph) cudaGraphExecDestroy(e->gexec);
    for (cudaEvent_t ev : e->join) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    for (spk_ctx* c : e->group) spk_ctx_destroy(c);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
    return SPK_OK;
}

extern "C" int spk_ensemble_create(const spk_params_t* boxes, int nbox, void* cuda_stream, spk_ensemble** out) {
    if (!boxes || nbox <= 0 || !out) return ens_fail("null argument or empty ensemble", SPK_ERR_ARG);
    *out = nullptr;
    for (int i = 0; i < nbox; i++) {
        const spk_params_t& p = boxes[i];
        if (p.closure)
            return ens_fail("ensemble box " + std::to_string(i) + ": the learned closure is not supported in ensembles",
                            SPK_ERR_UNSUPPORTED);
        if (p.shearing)
            return ens_fail("ensemble box " + std::to_string(i) + ": the shearing box is not supported in ensembles",
                            SPK_ERR_UNSUPPORTED);
        if (p.supertimestepping && !p.sts_every_step)
            return ens_fail("ensemble box " + std::to_string(i) +
                                ": super-time-stepping that alternates between steps is not supported in ensembles",
                            SPK_ERR_UNSUPPORTED);
    }
    // groups in order of first appearance
    std::vector<std::vector<int>> members;
    std::vector<std::pair<int, int>> where((size_t)nbox);
    for (int i = 0; i < nbox; i++) {
        int gidx = -1;
        for (size_t gq = 0; gq < members.size(); gq++)
            if (same_group(boxes[members[gq][0]], boxes[i])) { gidx = (int)gq; break; }
        if (gidx < 0) { gidx = (int)members.size(); members.emplace_back(); }
        where[(size_t)i] = {gidx, (int)members[(size_t)gidx].size()};
        members[(size_t)gidx].push_back(i);
    }
    spk_ensemble* e = new spk_ensemble();
    e->where = where;
    e->stream = (cudaStream_t)cuda_stream;
    if (!e->stream) {
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete e;
            return ens_fail("cudaStreamCreateWithFlags failed", SPK_ERR_CUDA);
        }
        e->own_stream = true;
    }
    if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
        spk_ensemble_destroy(e);
        return ens_fail("cudaEventCreate failed", SPK_ERR_CUDA);
    }
    for (size_t gq = 0; gq < members.size(); gq++) {
        std::vector<double> nu, nu_m, nu_th;
        for (int i : members[gq]) {
            nu.push_back(boxes[i].nu);
            nu_m.push_back(boxes[i].nu_m);
            nu_th.push_back(boxes[i].nu_th);
        }
        spk_ctx* c = nullptr;
        const int rc = ctx_create_group(boxes[members[gq][0]], nu, nu_m, nu_th, &c);
        if (rc != SPK_OK) {
            const std::string msg = "ensemble box " + std::to_string(members[gq][0]) + ": " + g_create_error;
            spk_ensemble_destroy(e);
            return ens_fail(msg, rc);
        }
        e->group.push_back(c);
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            spk_ensemble_destroy(e);
            return ens_fail("cudaEventCreate failed", SPK_ERR_CUDA);
        }
        e->join.push_back(ev);
    }
    *out = e;
    return SPK_OK;
}

extern "C" int spk_ensemble_size(const spk_ensemble* e, int* nbox, int* ngroups) {
    if (!e) return SPK_ERR_ARG;
    if (nbox) *nbox = (int)e->where.size();
    if (ngroups) *ngroups = (int)e->group.size();
    return SPK_OK;
}

static spk_ctx* ens_box(spk_ensemble* e, int i, int* b) {
    if (!e || i < 0 || i >= (int)e->where.size()) return nullptr;
    *b = e->where[(size_t)i].second;
    return e->group[(size_t)e->where[(size_t)i].first];
}

extern "C" int spk_ensemble_set_state(spk_ensemble* e, int i, const double* U, int where) {
    int b;
    spk_ctx* c = ens_box(e, i, &b);
    if (!c || !U) return ens_fail("ensemble box index out of range or null state", SPK_ERR_ARG);
    const size_t n = (size_t)c->F * c->nc;
    CK(cudaMemcpyAsync(c->U + (size_t)b * n, U, sizeof(double2) * n,
                       where ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream));
    c->dirty = true;
    return SPK_OK;
}

extern "C" int spk_ensemble_get_state(spk_ensemble* e, int i, double* U, int where) {
    int b;
    spk_ctx* c = ens_box(e, i, &b);
    if (!c || !U) return ens_fail("ensemble box index out of range or null state", SPK_ERR_ARG);
    const size_t n = (size_t)c->F * c->nc;
    CK(cudaMemcpyAsync(U, c->U + (size_t)b * n, sizeof(double2) * n,
                       where ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c->stream));
    if (where) CK(cudaStreamSynchronize(c->stream));
    return SPK_OK;
}

extern "C" int spk_ensemble_get_time(spk_ensemble* e, int i, double* t, double* dt, int* step) {
    int b;
    spk_ctx* c = ens_box(e, i, &b);
    if (!c) return ens_fail("ensemble box index out of range", SPK_ERR_ARG);
    const int rc = pull_scalars(c);
    if (rc) return rc;
    if (t) *t = c->h_sc[b].t;
    if (dt) *dt = c->h_sc[b].dt;
    if (step) *step = c->h_sc[b].step;
    return SPK_OK;
}

extern "C" int spk_ensemble_budgets(spk_ensemble* e, int i, spk_budgets_t* out) {
    int b;
    spk_ctx* c = ens_box(e, i, &b);
    if (!c || !out) return ens_fail("ensemble box index out of range or null output", SPK_ERR_ARG);
    return box_budgets(c, b, out);
}

extern "C" int spk_ensemble_advance(spk_ensemble* e, int nsteps) {
    if (!e || nsteps < 0) return SPK_ERR_ARG;
    if (nsteps == 0) return SPK_OK;
    // states set from outside are cleaned once (as spk_advance does), each
    // on its group stream, and the ensemble stream waits for the groups
    for (size_t gq = 0; gq < e->group.size(); gq++) {
        spk_ctx* c = e->group[gq];
        if (c->dirty) {
            launch_clean(c);
            const int rc = launch_status(c);
            if (rc) return ens_fail("ensemble group " + std::to_string(gq) + ": " + c->err, rc);
        }
        if (cudaEventRecord(e->join[gq], c->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->stream, e->join[gq], 0) != cudaSuccess)
            return ens_fail("ensemble stream ordering failed", SPK_ERR_CUDA);
    }
    if (!e->have_graph) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return ens_fail("ensemble graph capture failed to start", SPK_ERR_CUDA);
        cudaEventRecord(e->fork, e->stream);
        int bad = SPK_OK;
        std::string why;
        long launches = 0;
        for (size_t gq = 0; gq < e->group.size() && bad == SPK_OK; gq++) {
            spk_ctx* c = e->group[gq];
            cudaStreamWaitEvent(c->stream, e->fork, 0);      // the group stream joins the capture
            const long l0 = c->launches;
            record_step(c, 0);
            launches += c->launches - l0;
            c->kernels_per_step[0] = (int)(c->launches - l0);
            if (c->sticky) { bad = c->sticky; why = "ensemble group " + std::to_string(gq) + ": " + c->err; }
            cudaEventRecord(e->join[gq], c->stream);
            cudaStreamWaitEvent(e->stream, e->join[gq], 0);   // and joins back
        }
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (bad != SPK_OK || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return bad != SPK_OK ? ens_fail(why, bad)
                                 : ens_fail(std::string("ensemble graph capture: ") + cudaGetErrorString(ce), SPK_ERR_CUDA);
        }
        const cudaError_t ie = cudaGraphInstantiate(&e->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return ens_fail(std::string("ensemble graph instantiate: ") + cudaGetErrorString(ie), SPK_ERR_CUDA);
        e->have_graph = true;
        e->kernels_per_step = (int)launches;
    }
    for (int it = 0; it < nsteps; it++) {
        if (cudaGraphLaunch(e->gexec, e->stream) != cudaSuccess) return ens_fail("ensemble graph launch failed", SPK_ERR_CUDA);
        for (spk_ctx* c : e->group) c->h_step++;
    }
    // per-box calls after this (get_state, budgets) run on the group streams
    cudaEventRecord(e->fork, e->stream);
    for (spk_ctx* c : e->group) cudaStreamWaitEvent(c->stream, e->fork, 0);
    return SPK_OK;
}

extern "C" int spk_ensemble_synchronize(spk_ensemble* e) {
    if (!e) return SPK_ERR_ARG;
    const cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return ens_fail(std::string("ensemble: ") + cudaGetErrorString(ce), SPK_ERR_CUDA);
    for (size_t gq = 0; gq < e->group.size(); gq++) {
        spk_ctx* c = e->group[gq];
        const int rc = spk_synchronize(c);
        if (rc) return ens_fail("ensemble group " + std::to_string(gq) + ": " + c->err, rc);
    }
    return SPK_OK;
}

extern "C" int spk_ensemble_kernels_per_step(const spk_ensemble* e, int* kernels) {
    if (!e || !kernels) return SPK_ERR_ARG;
    *kernels = e->kernels_per_step;
    return SPK_OK;
}

extern "C" const char* spk_last_error(const spk_ctx* c) {
    return c ? c->err.c_str() : g_create_error.c_str();
}

// ---------------------------------------------------------------------------
// accounting and per-pass timing
// ---------------------------------------------------------------------------
struct PassBytes { double x_inv, y_inv, z, y_fwd, x_fwd, rhs[3]; };

// Algorithmic HBM bytes of each pass: every array the pass must read or
// write, once; products only where the 2/3 mask keeps them.
// masked_live: the deferred masked modes carry content (DevScalars::masked_live)
static PassBytes pass_bytes(const spk_ctx* c, bool masked_live = true) {
    PassBytes b;
    const double nc = (double)c->nc, b_t = (double)csize(c), s16 = 16.0;
    int nx_keep = 0, ny_keep = 0;
    for (int i = 0; i < c->nx; i++) nx_keep += c->mx[i] != 0.0;
    for (int j = 0; j < c->ny; j++) ny_keep += c->my[j] != 0.0;
    const double nkz = (double)c->nx * c->ny * c->kz_keep;          // after the z R2C
    const double nkyz = (double)c->nx * ny_keep * c->kz_keep;       // after the y forward
    const double nkxyz = (double)nx_keep * ny_keep * c->kz_keep;    // after the x forward
    const int nx_in = c->F + (c->aniso_rhs ? 1 : 0);                // x inverse outputs (gx extra)
    b.x_inv = c->F * nc * s16 + nx_in * nc * b_t;
    b.y_inv = nx_in * nc * b_t + c->nin * nc * b_t;
    b.z = c->nin * nc * b_t + c->nout * nkz * b_t;
    if (c->defer && !masked_live) {
        // trimmed inverse passes: only the kept (ky, kz) columns enter and
        // only kz < kz_keep leaves the x and y passes
        const double nyz = (double)c->nx * ny_keep * c->kz_keep;    // x inverse in and out
        const double nz_in = (double)c->nx * c->ny * c->kz_keep;      // y inverse out, z in
        b.x_inv = c->F * nyz * s16 + nx_in * nyz * b_t;
        b.y_inv = nx_in * nyz * b_t + c->nin * nz_in * b_t;
        b.z = c->nin * nz_in * b_t + c->nout * nkz * b_t;
    }
    b.y_fwd = c->nout * nkz * b_t + c->nout * nkyz * b_t;
    b.x_fwd = c->nout * nkyz * b_t + c->nout * nkxyz * b_t;
    const double nl = c->nout * nkxyz * b_t;
    if (c->defer) {
        // stages 0 and 1 touch the kept modes only; stage 2 also moves the
        // masked modes once (U r, U w)
        b.rhs[0] = nl + 3.0 * c->F * nkxyz * s16;
        b.rhs[1] = nl + 4.0 * c->F * nkxyz * s16;
        b.rhs[2] = nl + 3.0 * c->F * nkxyz * s16 + (masked_live ? 2.0 * c->F * (nc - nkxyz) * s16 : 0.0);
        return b;
    }
    b.rhs[0] = nl + 3.0 * c->F * nc * s16;    // U r, U w, S w
    b.rhs[1] = nl + 4.0 * c->F * nc * s16;    // U r, S r, U w, S w
    b.rhs[2] = nl + 3.0 * c->F * nc * s16;    // U r, S r, U w
    return b;
}

extern "C" int spk_step_info(spk_ctx* c, int* kps, double* bytes) {
    if (!c) return SPK_ERR_ARG;
    if (kps) {
        if (!c->have_graph[0] && !c->have_graph[1]) {
            // record (and discard) one step to count its launches
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            const long l0 = c->launches;
            record_step(c, c->h_step & 1);
            c->kernels_per_step[c->h_step & 1] = (int)(c->launches - l0);
            CK(cudaStreamEndCapture(c->stream, &g));
            cudaGraphDestroy(g);
        }
        *kps = std::max(c->kernels_per_step[0], c->kernels_per_step[1]);
    }
    if (bytes) {
        if (c->p.heat_equation) {
            *bytes = 3.0 * 3.0 * c->F * (double)c->nc * 16.0;
        } else {
            bool live = true;
            if (c->defer) {
                const int rc = pull_scalars(c);
                if (rc) return rc;
                live = false;
                for (int b2 = 0; b2 < c->nb; b2++) live = live || c->h_sc[b2].masked_live != 0;
            }
            const PassBytes b = pass_bytes(c, live);
            *bytes = 3.0 * (b.x_inv + b.y_inv + b.z + b.y_fwd + b.x_fwd) + b.rhs[0] + b.rhs[1] + b.rhs[2];
        }
    }
    return SPK_OK;
}

extern "C" int spk_profile_passes(spk_ctx* c, int reps, spk_pass_stat_t* out, int max_out, int* n_out) {
    if (!c || !out || reps < 1) return SPK_ERR_ARG;
    if (!c->p.incompressible) return fail(c, SPK_ERR_UNSUPPORTED, "pass profiling needs the incompressible module");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    if (c->dirty) launch_clean(c);   // refreshes the masked-content flag
    bool live = true;
    if (c->defer) {
        const int rc = pull_scalars(c);
        if (rc) return rc;
        live = false;
        for (int b2 = 0; b2 < c->nb; b2++) live = live || c->h_sc[b2].masked_live != 0;
    }
    const PassBytes pb = pass_bytes(c, live);
    TrimScope ts(c);   // time the passes as a step runs them
    // with deferred masked modes the RHS of stages 0-1 (kept modes) and of
    // stage 2 (kept modes + the step's masked modes) are timed apart
    const char* names[7] = {"x_inverse", "y_inverse", "z_products", "y_forward", "x_forward", "rhs_rk", "rhs_rk_01"};
    const double bytes[7] = {pb.x_inv, pb.y_inv, pb.z, pb.y_fwd, pb.x_fwd, pb.rhs[2], pb.rhs[1]};
    const int npass = c->defer ? 7 : 6;
    int n = 0;
    // one warm pipeline so every buffer holds stage data
    pass_x_inverse(c, c->U, true, 2);
    pass_y_inverse(c, true);
    pass_z_products(c, false);
    pass_y_forward(c, c->nout, c->bufA, c->bufB);
    pass_x_forward(c);
    for (int k = 0; k < npass && n < max_out; k++) {
        CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < reps; r++) {
            switch (k) {
                case 0: pass_x_inverse(c, c->U, true, 2); break;
                case 1: pass_y_inverse(c, true); break;
                case 2: pass_z_products(c, false); break;
                case 3: pass_y_forward(c, c->nout, c->bufA, c->bufB); break;
                case 4: pass_x_forward(c); break;
                case 5: { XfArgs x = xf_args(c, c->U, XM_RK2, false); rhs(c, x); } break;
                default: { XfArgs x = xf_args(c, c->U, XM_RK1, false); rhs(c, x); } break;
            }
        }
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        memset(out[n].name, 0, sizeof(out[n].name));
        strncpy(out[n].name, names[k], sizeof(out[n].name) - 1);
        out[n].ms = ms / reps;
        out[n].bytes = bytes[k];
        out[n].launches_per_step = (c->defer && k == 5) ? 1 : (k == 6 ? 2 : 3);
        n++;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_out) *n_out = n;
    return launch_status(c);
}

// ---------------------------------------------------------------------------
// RHS without any allocation (spk_compute_dfield_noalloc)
//
// Some callers cannot call cudaMalloc: code that runs while another
// component owns the device memory (a fixed pool, an embedding framework's
// allocator), real-time loops that must not take cudaMalloc's implicit
// device synchronisation, and code paths that must not fail for lack of
// memory after start-up.  For them the RHS is computed with every scratch
// array of the pipeline (pass buffers, wavevector tables, FFT twiddles,
// device scalars) carved out of one file-scope device array.  The array is
// part of the loaded library: every GPU that loads it holds these bytes
// until the process exits.
// ---------------------------------------------------------------------------
#define SPK_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[SPK_NOALLOC_SCRATCH_BYTES];
// Device addresses of g_noalloc_scratch, one per device.  In host code the
// array's name is only a stand-in: a kernel must receive this address.
static void* g_noalloc_ptr[SPK_NOALLOC_MAX_DEVICES];

static std::mutex g_noalloc_mutex;   // host threads making their first calls at once

// Once per device, with that device current: the scratch address (and,
// once per process, the tensor-map encoder).
static int noalloc_setup(int dev) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[dev]) return SPK_OK;
    spk_ctx* c = nullptr;   // errors go to spk_last_error(NULL)
    void* ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return fail(nullptr, SPK_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    g_noalloc_ptr[dev] = ptr;
    return SPK_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int spk_compute_dfield_noalloc(const spk_params_t* p, const double* Uin, double* dUout, void* cuda_stream) {
    if (!p || !Uin || !dUout) return fail(nullptr, SPK_ERR_ARG, "null argument");
    std::string why;
    int rc = check_params(p, why);
    if (rc != SPK_OK) return fail(nullptr, rc, why);
    if (p->closure)
        return fail(nullptr, SPK_ERR_UNSUPPORTED,
                    "spk_compute_dfield_noalloc has no learned-closure parameters: set closure = 0");
    if (p->shearing)
        return fail(nullptr, SPK_ERR_UNSUPPORTED,
                    "spk_compute_dfield_noalloc keeps no remap clock: the shearing box needs a context");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SPK_NOALLOC_MAX_DEVICES)
        return fail(nullptr, SPK_ERR_CUDA, "no usable current device");
    // The tables and starting scalars are copied from host memory that lives
    // only for the duration of the call, so a capture would record copies
    // from freed memory: a call on a capturing stream is refused.
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t e = cudaStreamIsCapturing(cuda_stream ? (cudaStream_t)cuda_stream : cudaStreamLegacy, &cs);
        if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            if (e != cudaSuccess) cudaGetLastError();
            return fail(nullptr, SPK_ERR_UNSUPPORTED,
                        "spk_compute_dfield_noalloc was called on a stream that is being captured; it copies "
                        "host tables and cannot be recorded");
        }
    }

    // a context on the host stack, bound to the scratch array (no device
    // or pinned allocation; the caller's stream, or the legacy stream)
    spk_ctx ctx{};
    spk_ctx* c = &ctx;
    c->sticky = 0; c->bad_job = false; c->bad_why = ""; c->user_U = nullptr; c->dirty = false;
    rc = ctx_init(c, p, cuda_stream ? cuda_stream : (void*)cudaStreamLegacy);
    if (rc != SPK_OK) return rc;
    c->num_sms = 148;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);

    const size_t cs = csize(c);
    c->g.nx = c->nx; c->g.ny = c->ny; c->g.nz = c->nz; c->g.nzh = c->nzh;
    c->g.nzs = pass_row(c->nzh, c->fp32);
    c->g.ncs = (size_t)c->nx * c->ny * c->g.nzs;
    c->g.kz_keep = c->kz_keep; c->g.nc = c->nc;
    const size_t ntab = 2 * ((size_t)c->nx + c->ny + c->nzh);
    const size_t ntw = (size_t)c->nx + c->ny + c->nz;
    const size_t o_tab = 0;
    const size_t o_tw = align256(o_tab + sizeof(double) * ntab);
    const size_t o_sc = align256(o_tw + cs * ntw);
    const size_t bufbytes = c->p.incompressible ? align256(cs * c->g.ncs * c->nbuf_ch) : 0;
    const size_t o_bufA = align256(o_sc + sizeof(DevScalars));
    const size_t o_bufB = o_bufA + bufbytes;
    const size_t need = o_bufB + bufbytes;
    if (need > (size_t)SPK_NOALLOC_SCRATCH_BYTES) {
        char msg[200];
        snprintf(msg, sizeof(msg), "grid %dx%dx%d needs %.1f MiB of scratch; spk_compute_dfield_noalloc holds %u MiB",
                 c->nx, c->ny, c->nz, need / 1048576.0, (unsigned)(SPK_NOALLOC_SCRATCH_BYTES >> 20));
        return fail(nullptr, SPK_ERR_UNSUPPORTED, msg);
    }
    rc = noalloc_setup(dev);
    if (rc != SPK_OK) return rc;
    char* base = (char*)g_noalloc_ptr[dev];
    double* t = (double*)(base + o_tab);
    double* m = t + c->nx + c->ny + c->nzh;
    c->d_tab = t;
    c->g.kx = t; c->g.ky = t + c->nx; c->g.kz = t + c->nx + c->ny;
    c->g.mx = m; c->g.my = m + c->nx; c->g.mz = m + c->nx + c->ny;
    c->g.shear = 0.0; c->g.csh = 0.0; c->g.shsc = nullptr;
    c->d_tw = base + o_tw;
    c->sc = (DevScalars*)(base + o_sc);
    c->bufA = c->p.incompressible ? base + o_bufA : nullptr;
    c->bufB = c->p.incompressible ? base + o_bufB : nullptr;

    // tables and twiddles (the array keeps the previous call's contents)
    std::vector<double> tab(ntab);
    std::copy(c->kx.begin(), c->kx.end(), tab.begin());
    std::copy(c->ky.begin(), c->ky.end(), tab.begin() + c->nx);
    std::copy(c->kz.begin(), c->kz.end(), tab.begin() + c->nx + c->ny);
    std::copy(c->mx.begin(), c->mx.end(), tab.begin() + ntab / 2);
    std::copy(c->my.begin(), c->my.end(), tab.begin() + ntab / 2 + c->nx);
    std::copy(c->mz.begin(), c->mz.end(), tab.begin() + ntab / 2 + c->nx + c->ny);
    CK(cudaMemcpyAsync(t, tab.data(), sizeof(double) * ntab, cudaMemcpyHostToDevice, c->stream));
    std::vector<double> tw, all;
    FftPlan* pls[3] = {&c->plan_x, &c->plan_y, &c->plan_z};
    size_t off = 0;
    for (int a = 0; a < 3; a++) {
        twiddles(pls[a]->n, tw);
        all.insert(all.end(), tw.begin(), tw.end());
        pls[a]->tw = (char*)c->d_tw + off * cs;
        off += pls[a]->n;
    }
    if (c->fp32) {
        std::vector<float> tf(all.begin(), all.end());
        CK(cudaMemcpyAsync(c->d_tw, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice, c->stream));
    } else {
        CK(cudaMemcpyAsync(c->d_tw, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, c->stream));
    }
    // what must start at zero: the device scalars and the pass buffers
    // the device scalars start at zero except the viscosities the RHS reads
    // (a copy from this stack record, no allocation)
    DevScalars sc0;
    memset(&sc0, 0, sizeof(sc0));
    sc0.nu = c->p.nu; sc0.nu_m = c->p.nu_m; sc0.nu_th = c->p.nu_th;
    // (a pageable-memory copy: staged before the call returns)
    CK(cudaMemcpyAsync(c->sc, &sc0, sizeof(DevScalars), cudaMemcpyHostToDevice, c->stream));
    if (bufbytes) CK(cudaMemsetAsync(base + o_bufA, 0, 2 * bufbytes, c->stream));

    rc = spk_compute_dfield(c, Uin, dUout);
    if (rc != SPK_OK) g_create_error = c->err;
    return rc;
}

#include "spk_closure_api.cu"
#include "spk_tune.cu"
#include "spk_io.cu"
#include "spk_transfer.cu"
