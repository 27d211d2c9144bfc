// spk_kernels.cu -- the fused SPOOKY passes for sm_100a.
//
// Reference = LorenzoLMP/spooky-git; each kernel names the reference
// kernels / functions whose arithmetic it fuses.
#include <cuda_runtime.h>
#include <math.h>

#include "spk_kernels.cuh"

namespace spk {

__device__ __forceinline__ double2 d2(double x, double y) { return make_double2(x, y); }
// i*k*x
__device__ __forceinline__ double2 ik_mul(double k, double2 x) { return d2(-k * x.y, k * x.x); }

template <typename T> __device__ __forceinline__ C2<T> from_d2(double2 v) { return mk<T>((T)v.x, (T)v.y); }
template <typename V> __device__ __forceinline__ double2 to_d2(V v) { return d2((double)v.x, (double)v.y); }

// Iteration bound of every mbarrier wait (a wait that runs out sets the
// error flag instead of hanging).
#define SPK_WAIT_ITERS (1u << 24)

// ---------------------------------------------------------------------------
// Block-wide maxima of n per-thread values (the CFL maxima of the z pass).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void warp_block_max(T* v, int n, T* red) {
    // v[0..n): per-thread values -> red[0..n) block maxima (all threads call)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int q = 0; q < n; q++) {
        T x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) red[q * 32 + w] = x;
    }
    __syncthreads();
    if (threadIdx.x < n) {
        T x = (T)0;
        for (int i = 0; i < nw; i++) x = fmax(x, red[threadIdx.x * 32 + i]);
        red[threadIdx.x * 32] = x;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Time-update helpers of the elementwise RHS kernel (k_rhs) and the heat mode.
// ---------------------------------------------------------------------------
// New state value of one mode (writes the RK scratch where the scheme needs
// it).  In XM_DFIELD mode R goes to the output array and X is returned.
__device__ __forceinline__ double2 step_value(const XfArgs& a, size_t gi, double2 X, double2 R, double dt) {
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
            const double2 S = a.S[gi];
            const double2 Un = d2(1.0 * S.x + bu * R.x, 1.0 * S.y + bu * R.y);
            a.S[gi] = d2(1.0 * Un.x + bs * R.x, 1.0 * Un.y + bs * R.y);
            return Un;
        }
        case XM_RK2: {
            const double bu = g2 * dt;
            const double2 S = a.S[gi];
            return d2(1.0 * S.x + bu * R.x, 1.0 * S.y + bu * R.y);
        }
        case XM_EULER:
            return d2(1.0 * X.x + dt * R.x, 1.0 * X.y + dt * R.y);
        default:
            a.out[gi] = R;
            return X;
    }
}

// CleanDivergence (cuda_kernels_generic.cu:288-313) of a 3-vector at one mode.
__device__ __forceinline__ void clean3(double2* V, double kx, double ky, double kz) {
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
    const double sx = kx * V[0].x + ky * V[1].x + kz * V[2].x;
    const double sy = kx * V[0].y + ky * V[1].y + kz * V[2].y;
    V[0] = d2(V[0].x - kx * ik2 * sx, V[0].y - kx * ik2 * sy);
    V[1] = d2(V[1].x - ky * ik2 * sx, V[1].y - ky * ik2 * sy);
    V[2] = d2(V[2].x - kz * ik2 * sx, V[2].y - kz * ik2 * sy);
}

// ---------------------------------------------------------------------------
// Heat-equation mode (spectral only): nablaOpScalar with flag 0
// (physics.cu:217-221) and the RK3 / Euler update.
// ---------------------------------------------------------------------------
__global__ void k_heat(const __grid_constant__ XfArgs a) {
    const size_t nc = a.g.nc;
    const bool sts = (a.sts_mask >> a.TH) & 1u;
    for (size_t gb = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gb < nc * a.nb; gb += (size_t)gridDim.x * blockDim.x) {
        const size_t box = gb / nc, gi = gb - box * nc;
        const double dt = a.sc[box].dt, nu_th = a.sc[box].nu_th;
        const size_t off = box * a.box_state + (size_t)a.TH * nc + gi;
        const int k = (int)(gi % a.g.nzh);
        const size_t r = gi / a.g.nzh;
        const int j = (int)(r % a.g.ny), i = (int)(r / a.g.ny);
        const double kx = a.g.kx[i], ky = a.g.ky[j], kz = a.g.kz[k];
        const double2 X = a.U[off];
        double2 R = d2(0.0, 0.0);
        if (!sts) {
            const double f = -nu_th * (kx * kx + ky * ky + kz * kz);
            R = d2(f * X.x, f * X.y);
        }
        const double2 Un = step_value(a, off, X, R, dt);
        if (a.mode != XM_DFIELD) a.U[off] = Un;
    }
}

// ---------------------------------------------------------------------------
// Fields::CleanFieldDivergence on the state (symmetries.cu:114-130).
// ---------------------------------------------------------------------------
// V: the vector field of box 0; box b's copy starts box_stride elements later.
__global__ void k_clean(DevGrid g, double2* V0, size_t box_stride, int nb) {
    const size_t nc = g.nc;
    const double shx = grid_shx(g);
    for (size_t gb = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gb < nc * nb; gb += (size_t)gridDim.x * blockDim.x) {
        const size_t box = gb / nc, gi = gb - box * nc;
        double2* V = V0 + box * box_stride;
        const int k = (int)(gi % g.nzh);
        const size_t r = gi / g.nzh;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        const double kx = g.kx[i] + shx * g.ky[j], ky = g.ky[j], kz = g.kz[k];
        double2 X[3] = {V[gi], V[nc + gi], V[2 * nc + gi]};
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
        const double sx = kx * X[0].x + ky * X[1].x + kz * X[2].x;
        const double sy = kx * X[0].y + ky * X[1].y + kz * X[2].y;
        const double kk[3] = {kx, ky, kz};
        for (int c = 0; c < 3; c++) V[c * nc + gi] = d2(X[c].x - kk[c] * ik2 * sx, X[c].y - kk[c] * ik2 * sy);
    }
}

// ---------------------------------------------------------------------------
// Per box: the squared L2 norms of the nf fields from V0 over all modes and
// over the modes outside the 2/3 mask (grid.y = box), then the flag of the
// deferred masked modes: live unless the masked norm is below 1e-13 of the
// whole (a masked field that small changes nothing at FP64 resolution
// whether or not its decay is applied).
// ---------------------------------------------------------------------------
__global__ void k_masked_scan(DevGrid g, const double2* V0, int nf, size_t box_stride, DevScalars* scs) {
    const int box = blockIdx.y;
    const size_t nc = g.nc;
    const double2* V = V0 + (size_t)box * box_stride;
    double sa = 0.0, sm = 0.0;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % g.nzh);
        const size_t r = gi / g.nzh;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        double v = 0.0;
        for (int f = 0; f < nf; f++) {
            const double2 x = V[(size_t)f * nc + gi];
            v += x.x * x.x + x.y * x.y;
        }
        sa += v;
        if (!(g.mx[i] != 0.0 && g.my[j] != 0.0 && g.mz[k] != 0.0)) sm += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sm += __shfl_xor_sync(0xffffffffu, sm, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&scs[box].scan_all, sa);
        atomicAdd(&scs[box].scan_masked, sm);
    }
}

__global__ void k_masked_flag(DevScalars* scs) {
    if (threadIdx.x != 0) return;
    DevScalars& s = scs[blockIdx.x];
    s.masked_live = (s.scan_masked <= 1e-26 * s.scan_all) ? 0 : 1;   // NaN keeps the full treatment
    s.scan_all = 0.0;
    s.scan_masked = 0.0;
}

// ---------------------------------------------------------------------------
// Shell spectrum of two fields (Spectrum1d, cuda_kernels_generic.cu:441-472):
// per mode p = w Re(U1/N conj(U2/N)), w = 2 for kz index > 0, into shell
// m = (int)(|k|/dk + 0.5); shells m >= nbins are left out (the reference adds
// them past the end of its array).  out[nbins] receives the Parseval sum
// (weight 1 at kz = 0 and at the Nyquist plane, 2 elsewhere): the mean of
// f1 f2 over the grid (twoFieldCorrelation).  Per-CTA shared-memory
// histograms, then atomics into out (summation order varies).
// ---------------------------------------------------------------------------
__global__ void k_spectrum(DevGrid g, const double2* U1, const double2* U2, int nbins, double dk, double inv_n,
                           double* out) {
    extern __shared__ double hist[];
    for (int m = threadIdx.x; m < nbins; m += blockDim.x) hist[m] = 0.0;
    __syncthreads();
    const size_t nc = g.nc;
    const int nzl = g.nz / 2;   // Nyquist plane index
    const double shx = grid_shx(g);
    double tot = 0.0;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % g.nzh);
        const size_t r = gi / g.nzh;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        const double2 a = U1[gi], b = U2[gi];
        const double pr = (a.x * inv_n) * (b.x * inv_n) + (a.y * inv_n) * (b.y * inv_n);
        const double p = k > 0 ? 2.0 * pr : pr;
        tot += (k > 0 && k != nzl) ? 2.0 * pr : pr;
        const double kx = g.kx[i] + shx * g.ky[j], ky = g.ky[j], kz = g.kz[k];
        const int m = (int)(sqrt(kx * kx + ky * ky + kz * kz) / dk + 0.5);
        if (m < nbins) atomicAdd(&hist[m], p);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[nbins], tot);
    __syncthreads();
    for (int m = threadIdx.x; m < nbins; m += blockDim.x)
        if (hist[m] != 0.0) atomicAdd(&out[m], hist[m]);
}

// ---------------------------------------------------------------------------
// compute_dt (compute_dt.cu:15-309) from the device maxima; the stage count
// and stage coefficients of the super-time-stepping cycle (rkl.cu:207-591).
// One thread per box.
// ---------------------------------------------------------------------------
__global__ void k_dt(const __grid_constant__ DtArgs a, DevScalars* scs) {
    // one block per box; the box's own viscosities come from its scalars
    if (threadIdx.x != 0) return;
    DevScalars* sc = scs + blockIdx.x;
    const double nu = sc->nu, nu_m = sc->nu_m, nu_th = sc->nu_th;
    double gamma_v = 0.0, gamma_th = 0.0, gamma_par = 0.0, gamma_b = 0.0, gamma_tmp, gamma_sts = 0.0;
    const double kxmax = a.kxmax, kymax = a.kymax, kzmax = a.kzmax;
    double current_dt = sc->dt;
    double dt_hyp = 0.0, dt_par = 0.0, dt_sts = 0.0;
    auto in_sts = [&](int f) { return (a.sts_pos_mask >> f) & 1u; };
    if (a.heat) {
        gamma_tmp = ((kxmax) * (kxmax) + kymax * kymax + kzmax * kzmax) * nu_th;
        if (!in_sts(a.TH)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        dt_par = a.cfl * a.cfl_par / gamma_par;
        dt_sts = a.cfl_par / gamma_sts;
        current_dt = dt_par;
    }
    if (a.incompressible) {
        const double maxfx = __longlong_as_double((long long)sc->maxbits[0]);
        const double maxfy = __longlong_as_double((long long)sc->maxbits[1]);
        const double maxfz = __longlong_as_double((long long)sc->maxbits[2]);
        // x rates with the shearing box's |tremap| ky_max (0 without it)
        const double kxs = kxmax + fabs(sc->tremap) * kymax;
        gamma_v = (kxs * maxfx + kymax * maxfy + kzmax * maxfz);
        if (a.rotating) gamma_v += fabs(a.omega) / a.safety_source;
        if (a.shearing) gamma_v += fabs(a.shear) / a.safety_source;
        gamma_tmp = kxs * kxs * nu;
        if (!in_sts(a.VX)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kymax * kymax * nu;
        if (!in_sts(a.VY)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kzmax * kzmax * nu;
        if (!in_sts(a.VZ)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        if (a.bous) {
            gamma_th += sqrt(fabs(a.N2)) / a.safety_source;
            if (a.aniso) {
                gamma_th += sqrt(fabs(a.OmegaT2)) / a.safety_source;
                gamma_tmp = (kxs * kxs + kymax * kymax + kzmax * kzmax) * (1. / a.reynolds_ani);
            } else {
                gamma_tmp = (kxs * kxs + kymax * kymax + kzmax * kzmax) * nu_th;
            }
            if (!in_sts(a.TH)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        }
        if (a.mhd) {
            const double maxbx = __longlong_as_double((long long)sc->maxbits[3]);
            const double maxby = __longlong_as_double((long long)sc->maxbits[4]);
            const double maxbz = __longlong_as_double((long long)sc->maxbits[5]);
            gamma_b = kxs * maxbx + kymax * maxby + kzmax * maxbz;
            gamma_tmp = kxs * kxs * nu_m;
            if (!in_sts(a.BX)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kymax * kymax * nu_m;
            if (!in_sts(a.BY)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kzmax * kzmax * nu_m;
            if (!in_sts(a.BZ)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        }
        if (a.closure) {
            // the learned closure's eddy viscosity and resistivity as parabolic rates
            const double k2 = kxmax * kxmax + kymax * kymax + kzmax * kzmax;
            gamma_par += k2 * __longlong_as_double((long long)sc->maxbits[6]);
            if (a.mhd) gamma_par += k2 * __longlong_as_double((long long)sc->maxbits[7]);
        }
        dt_hyp = a.cfl / (gamma_v + gamma_th + gamma_b);
        dt_par = a.cfl_par / gamma_par;
        dt_sts = a.cfl_sts / gamma_sts;
        current_dt = (dt_hyp < dt_par) ? dt_hyp : dt_par;
        if (a.sts) {
            if (current_dt > dt_sts * a.safety_sts) current_dt = dt_sts * a.safety_sts;
        }
    }
    if (a.with_fixed) current_dt = a.fixed_dt;
    const double t = sc->t;
    if (t + current_dt > a.t_final) current_dt = a.t_final - t;
    else if (t + current_dt - sc->t_lastsnap > a.toutput_flow) current_dt = a.toutput_flow - t + sc->t_lastsnap;
    if (a.sts) {
        if (dt_sts > current_dt) dt_sts = current_dt;
    }
    sc->dt = current_dt;
    sc->dt_hyp = dt_hyp;
    sc->dt_par = dt_par;
    sc->dt_sts = dt_sts;
    if (a.sts) {
        const int smax = min(a.rkl_smax, SPK_RKL_MAX - 1);
        const double scrh = current_dt / dt_sts;
        int s;
        if (a.sts_alg == STS_ALG_STS) {
            // RKLegendre::compute_cycle_STS (rkl.cu:207-283): n sub-steps
            // applied in the reverse order of the sequence, tau = ts[n - m - 1]
            s = (int)floor(sts_sub_steps(dt_sts, current_dt, SPK_STS_DAMPING) + 1.0);
            if (s > smax || s < 1) { sc->err = 1; s = min(max(s, 1), smax); }
            const double dtc = s > 1 ? sts_corrected_dt(s, current_dt, SPK_STS_DAMPING) : 0.0;
            for (int st = 1; st <= s; st++) {
                sc->rkl[st][0] = 1.0; sc->rkl[st][1] = 0.0;
                sc->rkl[st][2] = s > 1 ? sts_tau(dtc, s - st, s, SPK_STS_DAMPING) : current_dt;
                sc->rkl[st][3] = 0.0; sc->rkl[st][4] = 0.0;
            }
        } else if (a.sts_alg == STS_ALG_RKL1) {
            // RKLegendre::compute_cycle_RKL1 (rkl.cu:286-434)
            s = 1 + (int)(4.0 * scrh / (1.0 + sqrt(1.0 + 8.0 * scrh)));
            if (s > smax || s < 1) { sc->err = 1; s = min(max(s, 1), smax); }
            const double w1 = 2.0 / (s * s + s);
            sc->rkl[1][0] = 0.0; sc->rkl[1][1] = 0.0;
            sc->rkl[1][2] = w1 * current_dt;
            sc->rkl[1][3] = 0.0; sc->rkl[1][4] = 0.0;
            for (int st = 2; st <= s; st++) {
                const double mu_j = (2. * st - 1.) / st;
                sc->rkl[st][0] = mu_j;
                sc->rkl[st][1] = -(st - 1.) / st;
                sc->rkl[st][2] = current_dt * (w1 * mu_j);
                sc->rkl[st][3] = 0.0; sc->rkl[st][4] = 0.0;
            }
        } else {
            // RKLegendre::compute_cycle_RKL2 recurrences, FP64 (rkl.cu:467-494, 540-586)
            const double s_str = 4.0 * (1.0 + 2.0 * scrh) / (1.0 + sqrt(9.0 + 16.0 * scrh));
            s = 1 + (int)(s_str);
            if (s > smax || s < 1) { sc->err = 1; s = min(max(s, 1), smax); }
            const double w1 = 4.0 / (s * s + s - 2.0);
            double b_j, b_jm1, b_jm2, a_jm1;
            b_j = b_jm1 = b_jm2 = 1.0 / 3.0;
            a_jm1 = 1.0 - b_jm1;
            sc->rkl[1][0] = 0.0; sc->rkl[1][1] = 0.0;
            sc->rkl[1][2] = current_dt * (w1 / 3.0);
            sc->rkl[1][3] = 0.0; sc->rkl[1][4] = 0.0;
            for (int st = 2; st <= s; st++) {
                const double mu_j = (2. * st - 1.) / st * b_j / b_jm1;
                const double mu_tilde_j = w1 * mu_j;
                const double gamma_j = -a_jm1 * mu_tilde_j;
                const double nu_j = -(st - 1.) * b_j / (st * b_jm2);
                sc->rkl[st][0] = mu_j;
                sc->rkl[st][1] = nu_j;
                sc->rkl[st][2] = current_dt * mu_tilde_j;
                sc->rkl[st][3] = gamma_j * current_dt;
                sc->rkl[st][4] = (1.0 - mu_j - nu_j);
                b_jm2 = b_jm1;
                b_jm1 = b_j;
                a_jm1 = 1.0 - b_jm1;
                b_j = 0.5 * (st * st + 3.0 * st) / (st * st + 3.0 * st + 2);
            }
        }
        sc->s_rkl = s;
    }
    if (a.advance) {
        sc->t = t + current_dt;
        sc->step += 1;
    }
}

// ---------------------------------------------------------------------------
// Shearing box, end of a step (hydro_mhd_advance.cu:167-180): the remap
// clock advances by dt; past half a shear period it restarts from the new
// time (ShiftTime, shearing_remapping.cu:15-25) and the fields are remapped.
// ---------------------------------------------------------------------------
__global__ void k_shear_end(DevScalars* sc, double lx, double ly, double shear) {
    if (threadIdx.x != 0) return;
    double tr = sc->tremap + sc->dt;
    int remap = 0;
    if (tr > ly / (2.0 * shear * lx)) {
        tr = fmod(sc->t + ly / (2.0 * shear * lx), ly / (shear * lx)) - ly / (2.0 * shear * lx);
        remap = 1;
    }
    sc->tremap = tr;
    sc->remap = remap;
}

// RemapField (shearing_remapping.cu:27-46) of every field when the step
// remapped: mode (nx, ny) moves to nx + ny when that lies strictly inside
// (-NX/2, NX/2) (RemapComplexVec, cuda_kernels_generic.cu:386-412), every
// other destination is zero, then the 2/3 mask (MaskVector, :414-423).  A
// work item is one (field, y index, pair of kz columns): its x columns go to
// shared memory, then back gathered (destination nt takes source nt - ny),
// in place.
#define SPK_REMAP_KC 2
__global__ void k_remap(DevGrid g, double2* U, int F, const DevScalars* sc) {
    if (!sc->remap) return;
    extern __shared__ double2 col[];   // [nx][SPK_REMAP_KC]
    const int nx = g.nx, ny = g.ny, nzh = g.nzh;
    const int ngk = (nzh + SPK_REMAP_KC - 1) / SPK_REMAP_KC;
    const long items = (long)F * ny * ngk;
    const int lo = -(nx / 2), hi = nx - 1 - nx / 2;   // signed x indices
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const int kg = (int)(it % ngk);
        const long r = it / ngk;
        const int j = (int)(r % ny), f = (int)(r / ny);
        const int k0 = kg * SPK_REMAP_KC;
        double2* X = U + (size_t)f * g.nc;
        __syncthreads();   // the previous item's writes have read the columns
        for (int e = threadIdx.x; e < nx * SPK_REMAP_KC; e += blockDim.x) {
            const int i = e / SPK_REMAP_KC, k = k0 + e % SPK_REMAP_KC;
            if (k < nzh) col[e] = X[(size_t)k + (size_t)nzh * ((size_t)j + (size_t)ny * i)];
        }
        __syncthreads();
        const int nyv = (int)fmod((double)j + (ny / 2), (double)ny) - ny / 2;
        for (int e = threadIdx.x; e < nx * SPK_REMAP_KC; e += blockDim.x) {
            const int i = e / SPK_REMAP_KC, kk = e % SPK_REMAP_KC, k = k0 + kk;
            if (k >= nzh) continue;
            const int nt = (int)fmod((double)i + (nx / 2), (double)nx) - nx / 2;
            const int ns = nt - nyv;
            double2 v = make_double2(0.0, 0.0);
            if (nt > -(nx / 2) && nt < nx / 2 && ns >= lo && ns <= hi) {
                const int is = ns < 0 ? ns + nx : ns;
                const double m = g.mx[i] * g.my[j] * g.mz[k];
                const double2 s = col[is * SPK_REMAP_KC + kk];
                v = make_double2(s.x * m, s.y * m);
            }
            X[(size_t)k + (size_t)nzh * ((size_t)j + (size_t)ny * i)] = v;
        }
    }
}

// reset the dt maxima before the first stage of a step
__global__ void k_reset_max(DevScalars* sc) {
    if (threadIdx.x < 8) sc[blockIdx.x].maxbits[threadIdx.x] = 0ull;   // one block per box
}

// ---------------------------------------------------------------------------
// Super-time-stepping stage update shared by the spectral and the
// anisotropic variants:
//   STS  addReset, U <- U + tau dU (cuda_kernels_generic.cu:174-181);
//   RKL1 stage 1 (rkl.cu:360-377), then rkl1_stage (generic.cu:146-158);
//   RKL2 stage 1 (rkl.cu:515-532), then rkl2_stage (generic.cu:160-172).
// Stage 1 of RKL1 keeps U in Uc1 only: the reference's copies to Uc0 and
// dU0 are never read by that scheme.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rkl_update(const RklArgs& a, const double* c, size_t off, size_t gi, double2* Uc, double2 dU) {
    double2* Uc0 = a.Uc0 + off;
    double2* Uc1 = a.Uc1 + off;
    double2* dU0 = a.dU0 + off;
    const double2 U = Uc[gi];
    if (a.sts_alg == STS_ALG_STS) {
        Uc[gi] = d2(1.0 * U.x + c[2] * dU.x, 1.0 * U.y + c[2] * dU.y);
    } else if (a.stage == 1) {
        if (a.sts_alg == STS_ALG_RKL2) { Uc0[gi] = U; dU0[gi] = dU; }
        Uc1[gi] = U;
        Uc[gi] = d2(1.0 * U.x + c[2] * dU.x, 1.0 * U.y + c[2] * dU.y);
    } else if (a.sts_alg == STS_ALG_RKL1) {
        const double2 U1 = Uc1[gi];
        const double2 Y = d2(c[0] * U.x + c[1] * U1.x, c[0] * U.y + c[1] * U1.y);
        Uc1[gi] = U;
        Uc[gi] = d2(Y.x + c[2] * dU.x, Y.y + c[2] * dU.y);
    } else {
        const double2 U1 = Uc1[gi], U0 = Uc0[gi], D0 = dU0[gi];
        const double2 Y = d2(c[0] * U.x + c[1] * U1.x, c[0] * U.y + c[1] * U1.y);
        Uc1[gi] = U;
        Uc[gi] = d2(Y.x + c[4] * U0.x + c[2] * dU.x + c[3] * D0.x, Y.y + c[4] * U0.y + c[2] * dU.y + c[3] * D0.y);
    }
}

// STS variables with isotropic diffusion: nablaOpScalar (flag 0) + update.
__global__ void k_rkl_spectral(const __grid_constant__ RklArgs a, double2* U) {
    if (a.stage > a.sc->s_rkl) return;
    const double* c = a.sc->rkl[a.stage];
    const size_t nc = a.g.nc;
    const double shx = grid_shx(a.g);   // shearing box: the wavevector of the current remap clock
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % a.g.nzh);
        const size_t r = gi / a.g.nzh;
        const int j = (int)(r % a.g.ny), i = (int)(r / a.g.ny);
        const double kx = a.g.kx[i] + shx * a.g.ky[j], ky = a.g.ky[j], kz = a.g.kz[k];
        const double k2 = kx * kx + ky * ky + kz * kz;
        for (int v = 0; v < a.nsts; v++) {
            if (a.kind[v] == 3) continue;
            const double coef = a.kind[v] == 0 ? a.nu : (a.kind[v] == 1 ? a.nu_m : a.nu_th);
            double2* Uc = U + (size_t)a.fields[v] * nc;
            const double2 X = Uc[gi];
            const double f = -coef * k2;
            rkl_update(a, c, (size_t)v * nc, gi, Uc, d2(f * X.x, f * X.y));
        }
    }
}

// Anisotropic conduction STS stage: x-forward of the heat-flux channels,
// DivergenceMask (generic.cu:315-334) into dtheta, then the stage update.

// FP64 energy / dissipation sums with the half-spectrum weights
// (computeEnergy, spooky_output_functions.cu:23-55).
// fzh, fny: 32-bit dividers by nzh and ny (a box's modes, nx*ny*nzh, stay
// below 2^31 for every supported size), in place of 64-bit divisions that
// would bound the kernel by instruction issue
__global__ void k_budgets(DevGrid g, const double2* U, int F, double* sums, FastDiv fzh, FastDiv fny) {
    const double shx = grid_shx(g);
    const size_t nc = g.nc;
    __shared__ double red[2][32];
    for (int f = 0; f < F; f++) {
        double e = 0.0, d = 0.0;
        for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
            const unsigned r = fzh.div((unsigned)gi);
            const int k = (int)((unsigned)gi - r * (unsigned)g.nzh);
            const unsigned ui = fny.div(r);
            const int i = (int)ui, j = (int)(r - ui * (unsigned)g.ny);
            const double2 q = U[(size_t)f * nc + gi];
            const double w = k == 0 ? 1.0 : 2.0;
            const double a2 = q.x * q.x + q.y * q.y;
            const double kxs = g.kx[i] + shx * g.ky[j];
            const double k2 = kxs * kxs + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
            e += w * a2;
            d += w * k2 * a2;
        }
        for (int o = 16; o > 0; o >>= 1) { e += __shfl_xor_sync(0xffffffffu, e, o); d += __shfl_xor_sync(0xffffffffu, d, o); }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = e; red[1][threadIdx.x >> 5] = d; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double se = 0.0, sd = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) { se += red[0][w]; sd += red[1][w]; }
            atomicAdd(&sums[2 * f], se);
            atomicAdd(&sums[2 * f + 1], sd);
        }
        __syncthreads();
    }
}

}  // namespace spk
