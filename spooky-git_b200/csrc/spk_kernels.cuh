// spk_kernels.cuh -- argument blocks of the SPOOKY B200 passes.
//
// One RK3 stage is five passes over HBM (x = slowest axis, z = contiguous):
//   X-inverse  (k_axis, axis 0): FP64 state -> x-inverse-transformed channels
//              (+ divergence cleaning, + i*kx derivative channels, + 1/N^3)
//   Y-inverse  (k_axis, axis 1): -> (x, y, kz) channels (+ i*ky derivative)
//   Z          (k_zpass): z C2R of every channel line, real-space products
//              (Basdevant stress, u x B, u theta, anisotropic heat flux),
//              |u|,|B| maxima for dt, z R2C of the products (kz < kz_keep)
//   Y-forward  (k_axis, axis 1): products -> (x, ky, kz), kept ky rows only
//   X-forward  (k_xfwd): products -> (kx, ky, kz); the RHS (curls,
//              divergences, 2/3 mask, Boussinesq, diffusion, Leray) and the
//              low-storage RK3 / Euler update of the FP64 state.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <cuda.h>

#include <math.h>

#include "spk_fft.cuh"
#include "spk_tma.cuh"

namespace spk {

// Division by a runtime constant d >= 1 for x < 2^31: q = (umulhi(x, m) + x) >> l
// with l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1 (Granlund and
// Montgomery, PLDI 1994, round-up method).
struct FastDiv {
    unsigned m, l;
    __host__ __device__ inline unsigned div(unsigned x) const {
#ifdef __CUDA_ARCH__
        return (__umulhi(x, m) + x) >> l;
#else
        return (unsigned)(((unsigned long long)x * m >> 32) + x) >> l;
#endif
    }
    static FastDiv make(unsigned d) {
        FastDiv f;
        unsigned l = 0;
        while ((1ull << l) < d) l++;
        f.l = l;
        f.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
        return f;
    }
};

struct DevScalars;
struct DevGrid {
    int nx, ny, nz, nzh;
    int nzs;                        // row length of the pass buffers (nzh rounded up to even)
    int kz_keep;                    // kz index k is inside the 2/3 mask iff k < kz_keep
    size_t nc;                      // nx*ny*nzh (state modes per field)
    size_t ncs;                     // nx*ny*nzs (pass-buffer elements per channel)
    const double *kx, *ky, *kz;     // wavevector tables (exact reference expressions)
    const double *mx, *my, *mz;     // separable mask factors, 0.0 or 1.0
    // shearing box: kx of mode (i, j) is kx[i] + shear * (tremap + csh * dt) * ky[j]
    // with tremap and dt from *shsc (csh: the RK stage's offset; shear 0: off)
    double shear, csh;
    const DevScalars* shsc;
};

#define SPK_RKL_MAX 128

// Super-time-stepping algorithms (values of spk_params_t::sts_algorithm).
enum { STS_ALG_STS = 1, STS_ALG_RKL1 = 2, STS_ALG_RKL2 = 3 };
// STS_NU, the damping of the classic STS sub-step sequence (rkl.hpp:32)
#define SPK_STS_DAMPING 0.001

// Device-resident step scalars (written by k_dt, read by every update pass).
struct DevScalars {
    double t, dt, dt_hyp, dt_par, dt_sts, t_lastsnap;
    unsigned long long maxbits[8];  // bit patterns of max |ux| |uy| |uz| |bx| |by| |bz| nu_t eta_t
    int step, s_rkl, err, nonfinite;
    // stage j of the super-time-stepping cycle: U <- c0 U + c1 U1 + c2 dU + c3 dU0 + c4 U0
    // (RKL2: mu, nu, dt*mu~, dt*gamma, 1-mu-nu; RKL1: mu, nu, dt*mu~;
    // STS: the sub-step tau in c2)
    double rkl[SPK_RKL_MAX][5];
    double nu, nu_m, nu_th;         // this box's viscosity, resistivity, thermal diffusivity
    // deferred masked modes: 0 when the state's content outside the 2/3 mask
    // has an L2 norm below 1e-13 of the state's (rounding noise of a round
    // trip through real space; it only decays); set by k_masked_flag after a
    // state is set.  scan_*: the squared norms (scratch)
    int masked_live;
    double scan_all, scan_masked;
    // shearing box: the remap clock (TimeStepping::tremap) and whether the
    // step that just ended remapped the fields
    double tremap;
    int remap;
};

// ShearWavevector's tremap * shear (cuda_kernels_generic.cu:362-384) for
// the wavevector of the launch's stage; 0 without the shearing module.
__device__ __forceinline__ double grid_shx(const DevGrid& g) {
    if (g.shear == 0.0) return 0.0;
    return g.shear * (g.csh != 0.0 ? g.shsc->tremap + g.csh * g.shsc->dt : g.shsc->tremap);
}

// Classic super-time-stepping of Alexiades, Amiez & Gremaud (Commun. Numer.
// Meth. Eng. 12, 31, 1996) as the reference states it (rkl.cu:594-664).
// With a = (1 - sqrt(nu)) / (1 + sqrt(nu)) and c(N) = (1 - a^2N) / (1 + a^2N),
// N sub-steps of the damped Chebyshev sequence advance by
// dt_exp N c(N) / (2 sqrt(nu)) (their Eq. 2.10): sts_sub_steps solves that
// for N = dT by Newton's method from N = 1 (128 iterations, |dN| < 1e-5;
// -1 when it does not converge).
__host__ __device__ inline double sts_sub_steps(double dt_exp, double dT, double damping) {
    const double sq = sqrt(damping);
    const double a = (1.0 - sq) / (1.0 + sq);
    double N = 1.0;
    for (int it = 0; it < 128; it++) {
        const double b = pow(a, 2.0 * N);
        const double c = (1.0 - b) / (1.0 + b);
        const double db = 2.0 * log(a) * b;                       // d(a^2N)/dN
        const double dc = c - N * 2.0 / ((1.0 + b) * (1.0 + b)) * db;   // d(N c)/dN
        const double f = dT - 0.5 * dt_exp / sq * N * c;
        const double df = -0.5 * dt_exp / sq * dc;
        const double dN = f / df;
        N -= dN;
        if (fabs(dN) < 1.e-5) return N;
    }
    return -1.0;
}
// The explicit step that makes n sub-steps span dT exactly (STS_CorrectTimeStep).
__host__ __device__ inline double sts_corrected_dt(int n, double dT, double damping) {
    const double sq = sqrt(damping);
    const double a = (1.0 - sq) / (1.0 + sq);
    const double b = pow(a, 2.0 * n);
    const double c = (1.0 - b) / (1.0 + b);
    return dT * 2.0 * sq / (n * c);
}
// Sub-step i of n (STS_ComputeSubSteps, Eq. 2.9 of AAG).
__host__ __device__ inline double sts_tau(double dt_exp, int i, int n, double damping) {
    return dt_exp / ((-1.0 + damping) * cos(((2.0 * i + 1.0) * M_PI) / (2.0 * n)) + 1.0 + damping);
}
// Stage counts of one cycle for r = dt / dt_sts (rkl.cu:233-235, 324-327, 473-477).
__host__ __device__ inline int sts_stage_count(int alg, double r) {
    if (alg == STS_ALG_STS) return (int)floor(sts_sub_steps(1.0, r, SPK_STS_DAMPING) + 1.0);
    if (alg == STS_ALG_RKL1) return 1 + (int)(4.0 * r / (1.0 + sqrt(1.0 + 8.0 * r)));
    return 1 + (int)(4.0 * (1.0 + 2.0 * r) / (1.0 + sqrt(9.0 + 16.0 * r)));
}

#define SPK_MAXJOBS 16

// One channel of a strided-axis pass: a 4-D tensor map of the input array
// ([channel][x][y][k], k in scalars) and the output channel base.
struct AxisJob {
    alignas(64) CUtensorMap tm;
    void* out;
    int ch;         // channel coordinate of the input in its tensor map
    int in_state;   // input is the FP64 state (double2) instead of the pass type
    int deriv;      // multiply the input by i*k before the transform: 1 k along the axis (row n),
                    // 2 k of the outer index, 3 kz of the column
    int defer_grp;  // deferred masked modes: 1 velocity (nu), 2 magnetic field (nu_m), 0 none
    int hp;         // keep only |k|^2 > AxisArgs::hp_k2 (the small scales of the closure's variant 2)
    int pad_;
};

struct AxisArgs {
    DevGrid g;
    FftPlan plan;
    int axis;       // 0: x (tile = fixed j), 1: y (tile = fixed i)
    int kt;         // tile width (k columns, a power of two)
    int kcols;      // process columns [0, kcols)
    int row_filter; // store only rows whose mask factor along the axis is 1
    int outer_filter; // skip tiles whose outer index has mask factor 0 (no load, no store)
    int nb;           // boxes of the same geometry side by side (tile index includes the box)
    FastDiv fd_job, fd_box, fd_kb;   // tile -> job, box, outer index, k block (set by the launcher)
    int in_box_ch;    // channel offset between boxes in the input tensor map
    int out_box_ch;   // channel offset between boxes in the output buffer
    int box_rows;   // rows per TMA box (<= 256); N / box_rows boxes per tile
    int nst;        // pipeline stages
    int convert;    // input type differs from the pass type (FP64 state in the FP32 form)
    double scale;   // input scale factor
    const DevScalars* gate; // RKL stages: skip when gate_stage > gate->s_rkl
    int gate_stage;
    int* err;       // error word (set when a TMA wait runs out)
    // stage 1 or 2 of an RK3 step whose masked modes are deferred (XfArgs::defer):
    // the state's masked modes enter scaled by the stage's RK3 amplification
    int defer_stage;
    const DevScalars* scs;
    // trimmed inverse passes of a step whose state has no masked content
    // (DevScalars::masked_live == 0): 1 = x inverse (skip tiles of masked y
    // rows and of kz blocks past kz_keep), 2 = y inverse (skip kz blocks past
    // kz_keep; masked y rows, which the x inverse left unwritten, enter as 0)
    int trim;
    double hp_k2;           // high-pass threshold of the jobs with hp set
    // single-box trimmed pass: enumerate only the kept tiles (tr_outer: the
    // kept outer indices of the x inverse, tr_nkb k blocks below kz_keep)
    int tr_nouter, tr_nkb;
    const int* tr_outer;
    int tr_always;          // enumerate the kept tiles regardless of the flag (outer-filtered x forward)
    FastDiv tr_fd_job, tr_fd_box, tr_fd_kb;
    int njobs;
    AxisJob job[SPK_MAXJOBS];
};

enum ZMode { ZM_PRODUCTS = 0, ZM_INVERSE_ONLY = 1, ZM_RKL_FLUX = 2, ZM_TO_REAL = 3 };

struct ZArgs {
    DevGrid g;
    FftPlan plan;           // length nz
    int lines;              // lines per CTA
    int mode;
    const void* in; size_t cs_in; int nin;   // input channels (x, y, kz)
    void* out; size_t cs_out; int nout;      // output channels (x, y, kz) or real lines
    // input channel roles (-1 = absent); gz is derived from th in the pass
    int ch_u, ch_b, ch_th, ch_gx, ch_gy, derive_gz;
    // products
    int hydro, mhd, bous, aniso, sd;
    double chi, omegaT2;
    int do_max;
    unsigned long long* maxbits;
    int* nonfinite;
    int* err;               // set to 2 when a bulk copy never completed
    void* breal;            // real B lines [3][nx*ny*nz], pass precision
    int store_breal, load_breal;
    double* real_out;       // ZM_TO_REAL: [nin][nx*ny*nz] FP64
    const DevScalars* gate; // RKL stages: skip when gate_stage > gate->s_rkl
    int gate_stage;
    FastDiv fd_nz;          // division by NZ
    int nb;                 // boxes side by side: line index = box * nx*ny + line
    size_t in_box, out_box; // element offsets between boxes in `in` and `out`
    DevScalars* scs;        // per-box scalars (CFL maxima, non-finite flag)
    // learned closure: input channels ch_dx (d/dx of u [and B]) and ch_dy
    // (d/dy); d/dz derived in the pass from channels zder_src[] (appended
    // after the inputs); MLP parameters (SPK_CLOSURE_NPARAM floats)
    int trim;               // masked content absent: the kz >= kz_keep tail of every input row enters as 0
    int closure, ch_dx, ch_dy;
    int cl_grad9;           // closure variant 2: the 9 (18) gradient channels from ch_dx, [direction][component]
    int zder_n, zder_src[6];
    const float* cparams;
    float delta2;
    // diagnostics (general path only): 1 -- the symmetric matrix v_i v_j of
    // the vector at ch_u, components xx xy xz; 2 -- components yy yz zz
    int shear_part;
};

enum XMode { XM_RK0 = 0, XM_RK1 = 1, XM_RK2 = 2, XM_EULER = 3, XM_DFIELD = 4 };

struct XfArgs {
    DevGrid g;
    FftPlan plan;           // length nx
    int kt;
    const void* nl; size_t cs_nl;           // nonlinear channels after the y-forward pass
    int nl_T, nl_E, nl_F, nl_Q;             // first channel of each product group (-1 absent)
    double2* U; double2* S; double2* out;   // FP64 state, RK scratch, dfield output
    int F, VEL, MAG, TH;
    int incompressible, mhd, bous, heat, strat, sd, aniso_rhs;
    unsigned sts_mask;
    double nu, nu_m, nu_th, N2;
    int mode, clean;
    const DevScalars* sc;
    FastDiv fd_ny;          // division by ny (elementwise RHS kernel)
    FastDiv fd_nl;          // division by nx*ny: line index -> box
    int nb;                 // boxes side by side; sc points at nb DevScalars
    size_t box_state;       // F*nc: state elements per box (U, S, out)
    size_t box_nl;          // pass-buffer elements per box (products)
    // Deferred dealiased-out modes (HD/MHD RK3): stages 0 and 1 update only
    // the kept modes (a compact index over kxi x kyi x kz < kz_keep); stage 2
    // takes every mode, the masked ones through the RK3 amplification of
    // their linear (diffusive) right-hand side over the whole step.
    int defer;
    const int *kxi, *kyi;   // kept x and y indices
    int nkx, nky;
    FastDiv fd_kzk, fd_nky, fd_nkx;
    // shearing box (g.shear != 0): Coriolis force with rotating on
    int rotating;
    double omega;
};

struct RklArgs {
    DevGrid g;
    FftPlan plan;           // length nx (for the flux pass)
    int kt;
    const void* nl; size_t cs_nl;           // q channels after the y-forward pass
    double2* th;            // the STS variable(s) in the state
    double2 *Uc0, *Uc1, *dU0;
    int stage;              // 1..s
    int sts_alg;            // STS_ALG_*
    int nsts; int fields[8]; int kind[8];   // kind: 0 velocity(nu) 1 B(nu_m) 2 th iso(nu_th) 3 th aniso
    double nu, nu_m, nu_th;
    const DevScalars* sc;
};

struct DtArgs {
    int incompressible, heat, mhd, bous, aniso, sts, with_fixed;
    double kxmax, kymax, kzmax;
    double nu, nu_m, nu_th, reynolds_ani, N2, OmegaT2;
    double cfl, cfl_par, cfl_sts, safety_source, safety_sts;
    double t_final, toutput_flow, fixed_dt;
    unsigned sts_pos_mask;   // bit f set: field f in STS
    int VX, VY, VZ, BX, BY, BZ, TH;
    int advance;             // 1: t += dt, step += 1
    int rkl_smax;
    int sts_alg;             // STS_ALG_*
    int closure;             // add the closure's max eddy viscosity / resistivity (maxbits[6], [7])
    int shearing, rotating;  // the shearing box's rates (compute_dt.cu:110-121)
    double shear, omega;
};

}  // namespace spk
