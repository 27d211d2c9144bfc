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

// ---------------------------------------------------------------------------
// Strided-axis pass (x or y), persistent and pipelined.  Tile = one channel,
// one outer index, KT consecutive k columns, all N positions along the axis
// ([N][KT] in shared memory, the TMA box layout).  Thread 0 keeps nst tiles
// in flight with cp.async.bulk.tensor loads completing on per-stage
// mbarriers; the CTA transforms the oldest tile and stores it.  Fuses
// ComplexVecAssign + scaleKernel (cufft_routines.cu:23-39) and the i*k
// derivative of Gradient (cuda_kernels_generic.cu:249-260) into the
// pre-transform pass over shared memory.
// ---------------------------------------------------------------------------
#define SPK_WAIT_ITERS (1u << 24)

template <typename T, int DIR, int EPT>
__global__ void __launch_bounds__(256, 2) k_axis(const __grid_constant__ AxisArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if (a.gate && a.gate_stage > a.gate->s_rkl) return;
    const int N = a.plan.n, KT = a.kt, lkt = ilog2(KT), NST = a.nst;
    const int nel = N * KT;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int nouter = a.axis == 0 ? a.g.ny : a.g.nx;
    const int nkb = (a.kcols + KT - 1) / KT;
    const int total = a.njobs * nouter * nkb;
    const size_t in_elem = a.convert ? sizeof(double2) : sizeof(C2<T>);
    const size_t stage_bytes = ((size_t)nel * in_elem + 127) & ~(size_t)127;
    // 128-byte aligned base: NST barriers, then the stage buffers
    unsigned char* sbase = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase);
    unsigned char* stages = sbase + 128;
    C2<T>* wbuf = reinterpret_cast<C2<T>*>(stages + (size_t)NST * stage_bytes);   // when converting
    const double* kax = a.axis == 0 ? a.g.kx : a.g.ky;
    const double* max_ = a.axis == 0 ? a.g.mx : a.g.my;
    const size_t stride = a.axis == 0 ? (size_t)a.g.ny * a.g.nzs : (size_t)a.g.nzs;
    const uint32_t tile_bytes = (uint32_t)((size_t)nel * in_elem);
    const uint32_t box_bytes = tile_bytes / (uint32_t)(N / a.box_rows);

    auto issue = [&](int t, int s) {
        const int jb = t / (nouter * nkb);
        const int rem = t - jb * nouter * nkb;
        const int o = rem / nkb, kb = rem - o * nkb;
        const AxisJob& jo = a.job[jb];
        unsigned char* dst = stages + (size_t)s * stage_bytes;
        mbar_expect_tx(&bar[s], tile_bytes);
        for (int b = 0; b < N / a.box_rows; b++) {
            if (a.axis == 0) tma_load_4d(dst + (size_t)b * box_bytes, &jo.tm, &bar[s], 2 * kb * KT, o, b * a.box_rows, jo.ch);
            else             tma_load_4d(dst + (size_t)b * box_bytes, &jo.tm, &bar[s], 2 * kb * KT, b * a.box_rows, o, jo.ch);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < NST; s++) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < NST; s++) {
            const int t = blockIdx.x + s * gridDim.x;
            if (t < total) issue(t, s);
        }

    int i = 0;
    bool aborted = false;
    for (int t = blockIdx.x; t < total; t += gridDim.x, i++) {
        const int s = i % NST;
        const uint32_t par = (uint32_t)((i / NST) & 1);
        const bool ok = mbar_wait(&bar[s], par, SPK_WAIT_ITERS);
        if (__syncthreads_or(!ok)) { aborted = true; break; }
        const int jb = t / (nouter * nkb);
        const int rem = t - jb * nouter * nkb;
        const int o = rem / nkb, kb = rem - o * nkb;
        const AxisJob& jo = a.job[jb];
        const int k0 = kb * KT;
        const int kt = min(KT, a.kcols - k0);
        unsigned char* stg = stages + (size_t)s * stage_bytes;
        C2<T>* work;
        const int tn = t + NST * gridDim.x;
        if (a.convert) {
            // FP64 state -> pass type, with the scale and the derivative
            const double2* src = reinterpret_cast<const double2*>(stg);
#pragma unroll 4
            for (int u = 0; u < EPT; u++) {
                const int e = tid + u * nthr;
                if (e < nel) {
                    double2 x = src[e];
                    if (jo.deriv) x = ik_mul(kax[e >> lkt], x);
                    wbuf[e] = mk<T>((T)(x.x * a.scale), (T)(x.y * a.scale));
                }
            }
            __syncthreads();
            if (tid == 0 && tn < total) issue(tn, s);   // the stage was only read
            work = wbuf;
        } else {
            work = reinterpret_cast<C2<T>*>(stg);
            if (jo.deriv || a.scale != 1.0) {
                const T sc = (T)a.scale;
#pragma unroll 4
                for (int u = 0; u < EPT; u++) {
                    const int e = tid + u * nthr;
                    if (e < nel) {
                        C2<T> v = work[e];
                        if (jo.deriv) { const T kk = (T)kax[e >> lkt]; v = mk<T>(-kk * v.y, kk * v.x); }
                        work[e] = mk<T>(v.x * sc, v.y * sc);
                    }
                }
                __syncthreads();
            }
        }
        fft_run<T, DIR, EPT, true, 0>(work, KT, 1, KT, a.plan);
        size_t base = a.axis == 0 ? (size_t)o * a.g.nzs : (size_t)o * a.g.ny * a.g.nzs;
        C2<T>* out = (C2<T>*)jo.out + base + k0;
#pragma unroll 4
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            const int n = e >> lkt, col = e & (KT - 1);
            if (e < nel && col < kt && (!a.row_filter || max_[n] != 0.0))
                out[(size_t)n * stride + col] = work[e];
        }
        fence_proxy_async_smem();   // this thread's writes to the stage precede the next TMA fill
        __syncthreads();
        if (!a.convert && tid == 0 && tn < total) issue(tn, s);
    }
    if (aborted) {
        // a load never completed: report it, then give every stage a bounded
        // chance to drain before the shared memory is released
        if (tid == 0) {
            atomicExch(a.err, 2);
            for (int s = 0; s < NST; s++) mbar_wait(&bar[s], (uint32_t)(((i + s) / NST) & 1), SPK_WAIT_ITERS);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// z pass: a CTA owns `lines` (i,j) lines.  Input channels are paired into
// complex sequences Z = A + iB (Hermitian-extended, DC/Nyquist imaginary
// parts dropped), inverse-transformed, and the real-space products are
// formed point by point:
//   TracelessShearMatrix[MHD] (cuda_kernels.cu:39-55, 216-234),
//   MagneticEmf (:240-252), EnergyFluxVector (:277-289),
//   ComputeBGradTheta + ComputeAnisotropicHeatFlux (:360-383),
// with the |u|,|B| maxima of compute_dt (compute_dt.cu:82-101,196-210).
// The products are paired again, forward-transformed and unpacked into
// half spectra (the D2Z of each product), keeping kz < kz_keep.
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

template <typename T, int EPT>
__global__ void __launch_bounds__(256, 2) k_zpass(const __grid_constant__ ZArgs a) {
    if (a.gate && a.gate_stage > a.gate->s_rkl) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int NZ = a.g.nz, nzh = a.g.nzh, L = a.lines, NZp = padded_len(NZ);
    const int nlines = a.g.nx * a.g.ny;
    const int line0 = blockIdx.x * L;
    const int nl = min(L, nlines - line0);
    const int nin_all = a.nin + (a.derive_gz == 1 ? 1 : 0);
    const int npin = (nin_all + 1) / 2;
    const int npout = (a.nout + 1) / 2;
    C2<T>* inb = reinterpret_cast<C2<T>*>(smem_raw);
    C2<T>* outb = inb + (size_t)L * npin * NZp;
    const C2<T>* in = (const C2<T>*)a.in;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;

    // 1. a warp per (line, input pair): load both half spectra, build the
    //    Hermitian-extended paired sequence Z = A + iB
    auto chan_val = [&](int ch, size_t off, int k) -> C2<T> {
        if (ch < a.nin) {
            C2<T> v = in[(size_t)ch * a.cs_in + off];
            if (a.derive_gz == 2 && ch == a.ch_th) {   // this channel carries i*kz*theta
                const T kz = (T)a.g.kz[k];
                v = mk<T>(-kz * v.y, kz * v.x);
            }
            return v;
        }
        if (ch == a.nin && a.derive_gz == 1) {
            const C2<T> th = in[(size_t)a.ch_th * a.cs_in + off];
            const T kz = (T)a.g.kz[k];
            return mk<T>(-kz * th.y, kz * th.x);
        }
        return mk<T>((T)0, (T)0);
    };
    for (int lp = warp; lp < L * npin; lp += nwarp) {
        const int l = lp / npin, p = lp - l * npin;
        C2<T>* Z = inb + (size_t)lp * NZp;
        for (int k = lane; k < nzh; k += 32) {
            C2<T> A = mk<T>((T)0, (T)0), B = mk<T>((T)0, (T)0);
            if (l < nl) {
                const size_t off = (size_t)(line0 + l) * a.g.nzs + k;
                A = chan_val(2 * p, off, k);
                B = chan_val(2 * p + 1, off, k);
            }
            if (k == 0 || 2 * k == NZ) {
                Z[padi<1>(k)] = mk<T>(A.x, B.x);
            } else {
                Z[padi<1>(k)] = mk<T>(A.x - B.y, A.y + B.x);
                Z[padi<1>(NZ - k)] = mk<T>(A.x + B.y, B.x - A.y);
            }
        }
    }
    __syncthreads();
    fft_run<T, +1, EPT, false, 1>(inb, 1, NZp, L * npin, a.plan);

    auto val = [&](int l, int ch, int z) -> T {
        const C2<T> v = inb[(size_t)(l * npin + (ch >> 1)) * NZp + padi<1>(z)];
        return (ch & 1) ? v.y : v.x;
    };
    const int npts = L * NZ;
    const FastDiv fz = a.fd_nz;

    if (a.mode == ZM_TO_REAL) {
        for (int e = threadIdx.x; e < npts; e += blockDim.x) {
            const int l = (int)fz.div((unsigned)e), z = e - l * NZ;
            if (l >= nl) continue;
            const size_t line = (size_t)(line0 + l);
            for (int c = 0; c < a.nin; c++)
                a.real_out[((size_t)c * nlines + line) * NZ + z] = (double)val(l, c, z);
        }
        return;
    }

    // 2. real-space products
    T mu[6] = {(T)0, (T)0, (T)0, (T)0, (T)0, (T)0};
    int bad = 0;
    T* breal = (T*)a.breal;
    for (int e = threadIdx.x; e < npts; e += blockDim.x) {
        const int l = (int)fz.div((unsigned)e), z = e - l * NZ;
        // output channel ch of this point -> half of the paired complex slot
        T* orow = reinterpret_cast<T*>(outb + (size_t)l * npout * NZp + padi<1>(z));
        auto put = [&](int ch, T v) { orow[(size_t)(ch >> 1) * NZp * 2 + (ch & 1)] = v; };
        if (l >= nl) {
            for (int ch = 0; ch < 2 * npout; ch++) put(ch, (T)0);
            continue;
        }
        const size_t line = (size_t)(line0 + l);
        T ux = 0, uy = 0, uz = 0, bx = 0, by = 0, bz = 0, th = 0, gx = 0, gy = 0, gz = 0;
        if (a.ch_u >= 0) { ux = val(l, a.ch_u, z); uy = val(l, a.ch_u + 1, z); uz = val(l, a.ch_u + 2, z); }
        if (a.load_breal) {
            bx = breal[(0 * (size_t)nlines + line) * NZ + z];
            by = breal[(1 * (size_t)nlines + line) * NZ + z];
            bz = breal[(2 * (size_t)nlines + line) * NZ + z];
        } else if (a.ch_b >= 0) {
            bx = val(l, a.ch_b, z); by = val(l, a.ch_b + 1, z); bz = val(l, a.ch_b + 2, z);
        }
        if (a.ch_th >= 0 && a.derive_gz != 2) th = val(l, a.ch_th, z);
        if (a.ch_gx >= 0) gx = val(l, a.ch_gx, z);
        if (a.ch_gy >= 0) gy = val(l, a.ch_gy, z);
        if (a.derive_gz == 1) gz = val(l, a.nin, z);
        else if (a.derive_gz == 2) gz = val(l, a.ch_th, z);
        if (a.store_breal) {
            breal[(0 * (size_t)nlines + line) * NZ + z] = bx;
            breal[(1 * (size_t)nlines + line) * NZ + z] = by;
            breal[(2 * (size_t)nlines + line) * NZ + z] = bz;
        }
        if (a.do_max) {
            const T av[6] = {fabs(ux), fabs(uy), fabs(uz), fabs(bx), fabs(by), fabs(bz)};
#pragma unroll
            for (int q = 0; q < 6; q++) {
                if (!isfinite(av[q])) bad = 1;
                mu[q] = fmax(mu[q], av[q]);
            }
        }
        int q = 0;
        if (a.mode == ZM_PRODUCTS) {
            if (a.hydro) {
                if (!a.mhd) {
                    put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz) / (T)3.0);
                    put(1, ux * uy);
                    put(2, ux * uz);
                    put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz) / (T)3.0);
                    put(4, uy * uz);
                } else {
                    put(0, ((T)2.0 * ux * ux - uy * uy - uz * uz - (T)2.0 * bx * bx + by * by + bz * bz) / (T)3.0);
                    put(1, ux * uy - bx * by);
                    put(2, ux * uz - bx * bz);
                    put(3, (-ux * ux + (T)2.0 * uy * uy - uz * uz + bx * bx - (T)2.0 * by * by + bz * bz) / (T)3.0);
                    put(4, uy * uz - by * bz);
                }
                q = 5;
            }
            if (a.mhd) {
                put(q, -by * uz + bz * uy);
                put(q + 1, bx * uz - bz * ux);
                put(q + 2, -bx * uy + by * ux);
                q += 3;
            }
            if (a.bous) {
                put(q, ux * th); put(q + 1, uy * th); put(q + 2, uz * th);
                q += 3;
            }
        }
        if (a.aniso) {
            const T bgt = bx * gx + by * gy + bz * gz;
            const T b2 = bx * bx + by * by + bz * bz;
            const T bs = a.sd == 0 ? bx : (a.sd == 1 ? by : bz);
            const T chi = (T)a.chi, W = (T)a.omegaT2;
            put(q, chi * bx * (bgt + W * bs) / b2);
            put(q + 1, chi * by * (bgt + W * bs) / b2);
            put(q + 2, chi * bz * (bgt + W * bs) / b2);
            q += 3;
        }
        if (a.nout > 0 && (a.nout & 1)) put(a.nout, (T)0);
    }
    if (a.do_max) {
        __syncthreads();
        T* red = reinterpret_cast<T*>(outb + (size_t)L * npout * NZp);   // 6 x 32 scratch
        warp_block_max<T>(mu, 6, red);
        if (threadIdx.x < 6) {
            const double m = (double)red[threadIdx.x * 32];
            const unsigned long long bits = (unsigned long long)__double_as_longlong(m);
            unsigned long long* dst = a.maxbits + threadIdx.x;
            if (bits > *((volatile unsigned long long*)dst)) atomicMax(dst, bits);
        }
        if (bad) atomicOr(a.nonfinite, 1);
    }
    if (a.nout == 0) return;
    __syncthreads();
    fft_run<T, -1, EPT, false, 1>(outb, 1, NZp, L * npout, a.plan);

    // 3. a warp per (line, output pair): unpack the paired spectra (D2Z of
    //    each product), store kz < kz_keep
    const int kk = a.g.kz_keep;
    C2<T>* out = (C2<T>*)a.out;
    const T half = (T)0.5;
    for (int lp = warp; lp < L * npout; lp += nwarp) {
        const int l = lp / npout, p = lp - l * npout;
        if (l >= nl) continue;
        const C2<T>* Z = outb + (size_t)lp * NZp;
        const size_t off0 = (size_t)(line0 + l) * a.g.nzs;
        for (int k = lane; k < kk; k += 32) {
            const C2<T> zk = Z[padi<1>(k)], zm = Z[padi<1>(k ? NZ - k : 0)];
            out[(size_t)(2 * p) * a.cs_out + off0 + k] = mk<T>(half * (zk.x + zm.x), half * (zk.y - zm.y));
            if (2 * p + 1 < a.nout)
                out[(size_t)(2 * p + 1) * a.cs_out + off0 + k] = mk<T>(half * (zk.y + zm.y), half * (zm.x - zk.x));
        }
    }
}

// ---------------------------------------------------------------------------
// x-forward pass + RHS + time update.  Tile = fixed j, kt columns, all kx.
// Streams the product channels one at a time through shared memory; their
// k-weighted sums accumulate in registers:
//   NonLinHydroAdv (cuda_kernels.cu:82-98), MagneticShear (:257-272),
//   NonLinBoussinesqAdv (:293-304), DivergenceMask (generic.cu:315-334),
// then BoussinesqStrat (:310-325), nablaOpScalar (generic.cu:198-214),
// GradPseudoPressure (:128-159) and axpyComplex (generic.cu:137-144) of
// RungeKutta3 / ForwardEuler (hydro_mhd_advance.cu:79-248).
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

template <typename T, int EPT>
__global__ void __launch_bounds__(256, 2) k_xfwd(const __grid_constant__ XfArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C2<T>* buf = reinterpret_cast<C2<T>*>(smem_raw);
    const int N = a.g.nx, KT = a.kt, nzh = a.g.nzh;
    const size_t nc = a.g.nc;
    const int k0 = blockIdx.x * KT, j = blockIdx.y;
    const int kt = min(KT, nzh - k0);
    const size_t stride = (size_t)a.g.ny * nzh, base = (size_t)j * nzh;
    const double ky = a.g.ky[j], my = a.g.my[j];
    const bool nl_on = (my != 0.0) && (k0 < a.g.kz_keep);
    const double dt = a.sc->dt;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int nel = N * KT;
    const C2<T>* nl = (const C2<T>*)a.nl;

    const size_t nstride = (size_t)a.g.ny * a.g.nzs, nbase = (size_t)j * a.g.nzs + k0;   // pass buffers
    auto load_fft = [&](int ch) {
        const C2<T>* src = nl + (size_t)ch * a.cs_nl + nbase;
        C2<T> v[EPT];
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            const int n = e / KT, col = e - n * KT;
            v[u] = (e < nel && col < kt) ? src[(size_t)n * nstride + col] : mk<T>((T)0, (T)0);
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            if (e < nel) buf[e] = v[u];
        }
        __syncthreads();
        fft_run<T, -1, EPT, true, 0>(buf, KT, 1, KT, a.plan);
    };

    // u_strat of each mode of the tile (read before the velocity update),
    // for the theta group; only allocated with stratification
    double2* usd = reinterpret_cast<double2*>(smem_raw + (((size_t)nel * sizeof(C2<T>) + 15) & ~(size_t)15));

    // ---------------- velocity ----------------
    if (a.incompressible) {
        C2<T> acc[EPT][3];
#pragma unroll
        for (int u = 0; u < EPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = mk<T>((T)0, (T)0);
        if (nl_on && a.nl_T >= 0) {
            for (int c = 0; c < 5; c++) {
                load_fft(a.nl_T + c);
#pragma unroll
                for (int u = 0; u < EPT; u++) {
                    const int e = tid + u * nthr;
                    if (e < nel) {
                        const int n = e / KT, col = e - n * KT;
                        const C2<T> v = buf[e];
                        const T kx = (T)a.g.kx[n], kz = (T)a.g.kz[min(k0 + col, nzh - 1)], kyt = (T)ky;
                        switch (c) {
                            case 0: acc[u][0] = cadd(acc[u][0], cscale(kx, v)); acc[u][2] = csub(acc[u][2], cscale(kz, v)); break;
                            case 1: acc[u][0] = cadd(acc[u][0], cscale(kyt, v)); acc[u][1] = cadd(acc[u][1], cscale(kx, v)); break;
                            case 2: acc[u][0] = cadd(acc[u][0], cscale(kz, v)); acc[u][2] = cadd(acc[u][2], cscale(kx, v)); break;
                            case 3: acc[u][1] = cadd(acc[u][1], cscale(kyt, v)); acc[u][2] = csub(acc[u][2], cscale(kz, v)); break;
                            default: acc[u][1] = cadd(acc[u][1], cscale(kz, v)); acc[u][2] = cadd(acc[u][2], cscale(kyt, v)); break;
                        }
                    }
                }
                __syncthreads();
            }
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            if (e >= nel) continue;
            const int n = e / KT, col = e - n * KT;
            if (col >= kt) continue;
            const int k = k0 + col;
            const size_t gi = base + (size_t)n * stride + k;
            const double kx = a.g.kx[n], kz = a.g.kz[k];
            const double k2 = kx * kx + ky * ky + kz * kz;
            const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
            double2 X[3];
#pragma unroll
            for (int c = 0; c < 3; c++) X[c] = a.U[(size_t)(a.VEL + c) * nc + gi];
            const bool m = nl_on && a.g.mx[n] != 0.0 && a.g.mz[k] != 0.0;
            double2 R[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const double2 s = to_d2(acc[u][c]);
                R[c] = m ? d2(s.y, -s.x) : d2(0.0, 0.0);   // -i * mask * sum
            }
            if (a.strat) {
                const double2 th = a.U[(size_t)a.TH * nc + gi];
                if (a.sd == 0)      { R[0] = d2(R[0].x - th.x, R[0].y - th.y); usd[e] = X[0]; }
                else if (a.sd == 1) { R[1] = d2(R[1].x - th.x, R[1].y - th.y); usd[e] = X[1]; }
                else                { R[2] = d2(R[2].x - th.x, R[2].y - th.y); usd[e] = X[2]; }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (!((a.sts_mask >> (a.VEL + c)) & 1u)) {
                    const double f = -a.nu * k2;
                    R[c] = d2(R[c].x + f * X[c].x, R[c].y + f * X[c].y);
                }
            }
            // Leray: dU += i k (i k.dU)/k^2
            const double sx = kx * R[0].x + ky * R[1].x + kz * R[2].x;
            const double sy = kx * R[0].y + ky * R[1].y + kz * R[2].y;
            const double kk[3] = {kx, ky, kz};
#pragma unroll
            for (int c = 0; c < 3; c++) R[c] = d2(R[c].x - kk[c] * ik2 * sx, R[c].y - kk[c] * ik2 * sy);
            double2 Un[3];
#pragma unroll
            for (int c = 0; c < 3; c++) Un[c] = step_value(a, (size_t)(a.VEL + c) * nc + gi, X[c], R[c], dt);
            if (a.mode != XM_DFIELD) {
                // CleanFieldDivergence of the next step, applied to the new state
                if (a.clean) clean3(Un, kx, ky, kz);
#pragma unroll
                for (int c = 0; c < 3; c++) a.U[(size_t)(a.VEL + c) * nc + gi] = Un[c];
            }
        }
    }

    // ---------------- magnetic field ----------------
    if (a.mhd) {
        C2<T> acc[EPT][3];
#pragma unroll
        for (int u = 0; u < EPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = mk<T>((T)0, (T)0);
        if (nl_on && a.nl_E >= 0) {
            for (int c = 0; c < 3; c++) {
                load_fft(a.nl_E + c);
#pragma unroll
                for (int u = 0; u < EPT; u++) {
                    const int e = tid + u * nthr;
                    if (e < nel) {
                        const int n = e / KT, col = e - n * KT;
                        const C2<T> v = buf[e];
                        const T kx = (T)a.g.kx[n], kz = (T)a.g.kz[min(k0 + col, nzh - 1)], kyt = (T)ky;
                        switch (c) {
                            case 0: acc[u][1] = cadd(acc[u][1], cscale(kz, v)); acc[u][2] = csub(acc[u][2], cscale(kyt, v)); break;
                            case 1: acc[u][0] = csub(acc[u][0], cscale(kz, v)); acc[u][2] = cadd(acc[u][2], cscale(kx, v)); break;
                            default: acc[u][0] = cadd(acc[u][0], cscale(kyt, v)); acc[u][1] = csub(acc[u][1], cscale(kx, v)); break;
                        }
                    }
                }
                __syncthreads();
            }
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            if (e >= nel) continue;
            const int n = e / KT, col = e - n * KT;
            if (col >= kt) continue;
            const int k = k0 + col;
            const size_t gi = base + (size_t)n * stride + k;
            const double kx = a.g.kx[n], kz = a.g.kz[k];
            const double k2 = kx * kx + ky * ky + kz * kz;
            double2 X[3];
#pragma unroll
            for (int c = 0; c < 3; c++) X[c] = a.U[(size_t)(a.MAG + c) * nc + gi];
            const bool m = nl_on && a.g.mx[n] != 0.0 && a.g.mz[k] != 0.0;
            double2 Un[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const double2 s = to_d2(acc[u][c]);
                double2 R = m ? d2(-s.y, s.x) : d2(0.0, 0.0);   // i * mask * sum
                if (!((a.sts_mask >> (a.MAG + c)) & 1u)) {
                    const double f = -a.nu_m * k2;
                    R = d2(R.x + f * X[c].x, R.y + f * X[c].y);
                }
                Un[c] = step_value(a, (size_t)(a.MAG + c) * nc + gi, X[c], R, dt);
            }
            if (a.mode != XM_DFIELD) {
                if (a.clean) clean3(Un, kx, ky, kz);
#pragma unroll
                for (int c = 0; c < 3; c++) a.U[(size_t)(a.MAG + c) * nc + gi] = Un[c];
            }
        }
    }

    // ---------------- temperature ----------------
    if (a.bous) {
        C2<T> acc[EPT][2];
#pragma unroll
        for (int u = 0; u < EPT; u++) acc[u][0] = acc[u][1] = mk<T>((T)0, (T)0);
        const bool th_sts = (a.sts_mask >> a.TH) & 1u;
        if (nl_on) {
            for (int g = 0; g < 2; g++) {
                const int first = g == 0 ? a.nl_F : (a.aniso_rhs ? a.nl_Q : -1);
                if (first < 0) continue;
                for (int c = 0; c < 3; c++) {
                    load_fft(first + c);
#pragma unroll
                    for (int u = 0; u < EPT; u++) {
                        const int e = tid + u * nthr;
                        if (e < nel) {
                            const int n = e / KT, col = e - n * KT;
                            const C2<T> v = buf[e];
                            const T kc = c == 0 ? (T)a.g.kx[n] : (c == 1 ? (T)ky : (T)a.g.kz[min(k0 + col, nzh - 1)]);
                            acc[u][g] = cadd(acc[u][g], cscale(kc, v));
                        }
                    }
                    __syncthreads();
                }
            }
        }
#pragma unroll
        for (int u = 0; u < EPT; u++) {
            const int e = tid + u * nthr;
            if (e >= nel) continue;
            const int n = e / KT, col = e - n * KT;
            if (col >= kt) continue;
            const int k = k0 + col;
            const size_t gi = base + (size_t)n * stride + k;
            const double kx = a.g.kx[n], kz = a.g.kz[k];
            const double k2 = kx * kx + ky * ky + kz * kz;
            const double2 X = a.U[(size_t)a.TH * nc + gi];
            const bool m = nl_on && a.g.mx[n] != 0.0 && a.g.mz[k] != 0.0;
            const double2 s0 = to_d2(acc[u][0]);
            double2 R = m ? d2(s0.y, -s0.x) : d2(0.0, 0.0);   // -i * mask * k.(u theta)
            if (a.strat) { const double2 us = usd[e]; R = d2(R.x + a.N2 * us.x, R.y + a.N2 * us.y); }
            if (!th_sts) {
                if (a.aniso_rhs) {
                    const double2 s1 = to_d2(acc[u][1]);
                    if (m) R = d2(R.x - s1.y, R.y + s1.x);      // += i * mask * k.q
                } else {
                    const double f = -a.nu_th * k2;
                    R = d2(R.x + f * X.x, R.y + f * X.y);
                }
            }
            const double2 Un = step_value(a, (size_t)a.TH * nc + gi, X, R, dt);
            if (a.mode != XM_DFIELD) a.U[(size_t)a.TH * nc + gi] = Un;
        }
    }
}

// ---------------------------------------------------------------------------
// Heat-equation mode (spectral only): nablaOpScalar with flag 0
// (physics.cu:217-221) and the RK3 / Euler update.
// ---------------------------------------------------------------------------
__global__ void k_heat(const __grid_constant__ XfArgs a) {
    const size_t nc = a.g.nc;
    const double dt = a.sc->dt;
    const bool sts = (a.sts_mask >> a.TH) & 1u;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % a.g.nzh);
        const size_t r = gi / a.g.nzh;
        const int j = (int)(r % a.g.ny), i = (int)(r / a.g.ny);
        const double kx = a.g.kx[i], ky = a.g.ky[j], kz = a.g.kz[k];
        const double2 X = a.U[(size_t)a.TH * nc + gi];
        double2 R = d2(0.0, 0.0);
        if (!sts) {
            const double f = -a.nu_th * (kx * kx + ky * ky + kz * kz);
            R = d2(f * X.x, f * X.y);
        }
        const double2 Un = step_value(a, (size_t)a.TH * nc + gi, X, R, dt);
        if (a.mode != XM_DFIELD) a.U[(size_t)a.TH * nc + gi] = Un;
    }
}

// ---------------------------------------------------------------------------
// Fields::CleanFieldDivergence on the state (symmetries.cu:114-130).
// ---------------------------------------------------------------------------
__global__ void k_clean(DevGrid g, double2* V) {
    const size_t nc = g.nc;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % g.nzh);
        const size_t r = gi / g.nzh;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        const double kx = g.kx[i], ky = g.ky[j], kz = g.kz[k];
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
// compute_dt (compute_dt.cu:15-309) from the device maxima; RKL2 stage count
// and stage coefficients (rkl.cu:467-494, 540-586).  One thread.
// ---------------------------------------------------------------------------
__global__ void k_dt(const __grid_constant__ DtArgs a, DevScalars* sc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double gamma_v = 0.0, gamma_th = 0.0, gamma_par = 0.0, gamma_b = 0.0, gamma_tmp, gamma_sts = 0.0;
    const double kxmax = a.kxmax, kymax = a.kymax, kzmax = a.kzmax;
    double current_dt = sc->dt;
    double dt_hyp = 0.0, dt_par = 0.0, dt_sts = 0.0;
    auto in_sts = [&](int f) { return (a.sts_pos_mask >> f) & 1u; };
    if (a.heat) {
        gamma_tmp = ((kxmax) * (kxmax) + kymax * kymax + kzmax * kzmax) * a.nu_th;
        if (!in_sts(a.TH)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        dt_par = a.cfl * a.cfl_par / gamma_par;
        dt_sts = a.cfl_par / gamma_sts;
        current_dt = dt_par;
    }
    if (a.incompressible) {
        const double maxfx = __longlong_as_double((long long)sc->maxbits[0]);
        const double maxfy = __longlong_as_double((long long)sc->maxbits[1]);
        const double maxfz = __longlong_as_double((long long)sc->maxbits[2]);
        gamma_v = ((kxmax + 0.0 * kymax) * maxfx + kymax * maxfy + kzmax * maxfz);
        gamma_tmp = (kxmax) * (kxmax) * a.nu;
        if (!in_sts(a.VX)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kymax * kymax * a.nu;
        if (!in_sts(a.VY)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kzmax * kzmax * a.nu;
        if (!in_sts(a.VZ)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        if (a.bous) {
            gamma_th += sqrt(fabs(a.N2)) / a.safety_source;
            if (a.aniso) {
                gamma_th += sqrt(fabs(a.OmegaT2)) / a.safety_source;
                gamma_tmp = ((kxmax) * (kxmax) + kymax * kymax + kzmax * kzmax) * (1. / a.reynolds_ani);
            } else {
                gamma_tmp = ((kxmax) * (kxmax) + kymax * kymax + kzmax * kzmax) * a.nu_th;
            }
            if (!in_sts(a.TH)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        }
        if (a.mhd) {
            const double maxbx = __longlong_as_double((long long)sc->maxbits[3]);
            const double maxby = __longlong_as_double((long long)sc->maxbits[4]);
            const double maxbz = __longlong_as_double((long long)sc->maxbits[5]);
            gamma_b = (kxmax) * maxbx + kymax * maxby + kzmax * maxbz;
            gamma_tmp = (kxmax) * (kxmax) * a.nu_m;
            if (!in_sts(a.BX)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kymax * kymax * a.nu_m;
            if (!in_sts(a.BY)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kzmax * kzmax * a.nu_m;
            if (!in_sts(a.BZ)) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
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
        // RKLegendre::compute_cycle_RKL2 recurrences, FP64 (rkl.cu:467-494, 540-586)
        const double scrh = current_dt / dt_sts;
        const double s_str = 4.0 * (1.0 + 2.0 * scrh) / (1.0 + sqrt(9.0 + 16.0 * scrh));
        int s = 1 + (int)(s_str);
        if (s > a.rkl_smax || s > SPK_RKL_MAX - 1 || s < 1) { sc->err = 1; s = min(max(s, 1), min(a.rkl_smax, SPK_RKL_MAX - 1)); }
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
        sc->s_rkl = s;
    }
    if (a.advance) {
        sc->t = t + current_dt;
        sc->step += 1;
    }
}

// reset the dt maxima before the first stage of a step
__global__ void k_reset_max(DevScalars* sc) {
    if (threadIdx.x < 8) sc->maxbits[threadIdx.x] = 0ull;
}

// ---------------------------------------------------------------------------
// RKL2 stage update shared by the spectral and the anisotropic variants
// (rkl.cu:515-532 for stage 1, rkl2_stage generic.cu:160-172 for j >= 2).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rkl_update(const RklArgs& a, const double* c, size_t off, size_t gi, double2* Uc, double2 dU) {
    double2* Uc0 = a.Uc0 + off;
    double2* Uc1 = a.Uc1 + off;
    double2* dU0 = a.dU0 + off;
    if (a.stage == 1) {
        const double2 U = Uc[gi];
        Uc0[gi] = U;
        dU0[gi] = dU;
        Uc1[gi] = U;
        Uc[gi] = d2(1.0 * U.x + c[2] * dU.x, 1.0 * U.y + c[2] * dU.y);
    } else {
        const double2 U = Uc[gi], U1 = Uc1[gi], U0 = Uc0[gi], D0 = dU0[gi];
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
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % a.g.nzh);
        const size_t r = gi / a.g.nzh;
        const int j = (int)(r % a.g.ny), i = (int)(r / a.g.ny);
        const double kx = a.g.kx[i], ky = a.g.ky[j], kz = a.g.kz[k];
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
template <typename T, int EPT>
__global__ void __launch_bounds__(256, 2) k_xfwd_rkl(const __grid_constant__ RklArgs a, double2* U, int vslot) {
    if (a.stage > a.sc->s_rkl) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C2<T>* buf = reinterpret_cast<C2<T>*>(smem_raw);
    const double* cf = a.sc->rkl[a.stage];
    const int N = a.g.nx, KT = a.kt, nzh = a.g.nzh;
    const size_t nc = a.g.nc;
    const int k0 = blockIdx.x * KT, j = blockIdx.y;
    const int kt = min(KT, nzh - k0);
    const size_t stride = (size_t)a.g.ny * nzh, base = (size_t)j * nzh;
    const double ky = a.g.ky[j], my = a.g.my[j];
    const bool nl_on = (my != 0.0) && (k0 < a.g.kz_keep);
    const int nthr = blockDim.x, tid = threadIdx.x, nel = N * KT;
    const C2<T>* nl = (const C2<T>*)a.nl;
    C2<T> acc[EPT];
#pragma unroll
    for (int u = 0; u < EPT; u++) acc[u] = mk<T>((T)0, (T)0);
    const size_t nstride = (size_t)a.g.ny * a.g.nzs, nbase = (size_t)j * a.g.nzs + k0;   // pass buffers
    if (nl_on) {
        for (int c = 0; c < 3; c++) {
            const C2<T>* src = nl + (size_t)c * a.cs_nl + nbase;
            for (int e = tid; e < nel; e += nthr) {
                const int n = e / KT, col = e - n * KT;
                buf[e] = (col < kt) ? src[(size_t)n * nstride + col] : mk<T>((T)0, (T)0);
            }
            __syncthreads();
            fft_run<T, -1, EPT, true, 0>(buf, KT, 1, KT, a.plan);
#pragma unroll
            for (int u = 0; u < EPT; u++) {
                const int e = tid + u * nthr;
                if (e < nel) {
                    const int n = e / KT, col = e - n * KT;
                    const T kc = c == 0 ? (T)a.g.kx[n] : (c == 1 ? (T)ky : (T)a.g.kz[min(k0 + col, nzh - 1)]);
                    acc[u] = cadd(acc[u], cscale(kc, buf[e]));
                }
            }
            __syncthreads();
        }
    }
    double2* Uc = U + (size_t)a.fields[vslot] * nc;
#pragma unroll
    for (int u = 0; u < EPT; u++) {
        const int e = tid + u * nthr;
        if (e >= nel) continue;
        const int n = e / KT, col = e - n * KT;
        if (col >= kt) continue;
        const int k = k0 + col;
        const size_t gi = base + (size_t)n * stride + k;
        const bool m = nl_on && a.g.mx[n] != 0.0 && a.g.mz[k] != 0.0;
        const double2 s = to_d2(acc[u]);
        const double2 dU = m ? d2(-s.y, s.x) : d2(0.0, 0.0);   // i * mask * k.q
        rkl_update(a, cf, (size_t)vslot * nc, gi, Uc, dU);
    }
}

// FP64 energy / dissipation sums with the half-spectrum weights
// (computeEnergy, spooky_output_functions.cu:23-55).
__global__ void k_budgets(DevGrid g, const double2* U, int F, double* sums) {
    const size_t nc = g.nc;
    __shared__ double red[2][32];
    for (int f = 0; f < F; f++) {
        double e = 0.0, d = 0.0;
        for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
            const int k = (int)(gi % g.nzh);
            const size_t r = gi / g.nzh;
            const int j = (int)(r % g.ny), i = (int)(r / g.ny);
            const double2 q = U[(size_t)f * nc + gi];
            const double w = k == 0 ? 1.0 : 2.0;
            const double a2 = q.x * q.x + q.y * q.y;
            const double k2 = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
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
