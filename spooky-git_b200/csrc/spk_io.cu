// spk_io.cu -- real-space state and snapshot files (included by spk_api.cu).
//
// The reference's data files hold the real fields (src/io/hdf5_io.cu:19-111,
// written after Supervisor::Complex2RealFields) and a restart reads them
// back and transforms them to spectral space (hdf5_io.cu:114-252, then the
// R2C of Fields::allocate_and_move_to_gpu).  Here both transforms run on the
// device as plain FP64 discrete Fourier transforms, one CTA per line, using
// the context's RK scratch array S as the staging area (S carries nothing
// from one step to the next).  They run once per snapshot, not per step, so
// a direct O(N^2) sum per line is used: it is exact to FP64 rounding for
// every supported length and needs no plan.  The pass kernels of the step
// are not involved.

// DFT of one line of n complex values held in shared memory, output m:
// sum_p x[p] w^(m p mod n), w = e^(sign 2 pi i / n), summed in FP64.
__device__ __forceinline__ double2 line_dft_at(const double2* x, const double2* w, int n, int m) {
    double re = 0.0, im = 0.0;
    int q = 0;
    for (int p = 0; p < n; p++) {
        const double2 a = x[p], t = w[q];
        re += a.x * t.x - a.y * t.y;
        im += a.x * t.y + a.y * t.x;
        q += m;
        if (q >= n) q -= n;
    }
    return make_double2(re, im);
}

__device__ __forceinline__ void line_twiddles(double2* w, int n, double sign) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)q / (double)n, &s, &c);
        w[q] = make_double2(c, sign * s);
    }
}

// In-place complex DFT along one axis of a [F][nx][ny][nzh] array.  Line L
// starts at (L / d1) * s1 + ((L % d1) / d2) * s2 + (L % d2) * s3 and its
// elements are `stride` apart.
__global__ void k_line_dft(double2* A, long nlines, int n, long stride, long d1, long s1, long d2, long s2, long s3,
                           double sign) {
    extern __shared__ double2 io_sm[];
    double2* x = io_sm;
    double2* w = io_sm + n;
    line_twiddles(w, n, sign);
    for (long L = blockIdx.x; L < nlines; L += gridDim.x) {
        const long base = (L / d1) * s1 + ((L % d1) / d2) * s2 + (L % d2) * s3;
        __syncthreads();
        for (int p = threadIdx.x; p < n; p += blockDim.x) x[p] = A[base + p * stride];
        __syncthreads();
        for (int m = threadIdx.x; m < n; m += blockDim.x) A[base + m * stride] = line_dft_at(x, w, n, m);
    }
}

// Real lines of nz values (R, contiguous lines) -> their nz/2+1 lowest
// modes (U, lines nzh apart): the unnormalised R2C of cuFFT's D2Z.
__global__ void k_z_r2c(const double* R, double2* U, long nlines, int nz, int nzh) {
    extern __shared__ double2 io_sm[];
    double2* x = io_sm;
    double2* w = io_sm + nz;
    line_twiddles(w, nz, -1.0);
    for (long L = blockIdx.x; L < nlines; L += gridDim.x) {
        __syncthreads();
        for (int p = threadIdx.x; p < nz; p += blockDim.x) x[p] = make_double2(R[L * nz + p], 0.0);
        __syncthreads();
        for (int k = threadIdx.x; k < nzh; k += blockDim.x) U[L * nzh + k] = line_dft_at(x, w, nz, k);
    }
}

// Half spectra of nzh modes (lines nzh apart, in place) -> nz real values
// each, times `scale`, written over the same line as 2*nzh doubles (the
// reference's padded real layout).  The missing modes are the conjugates of
// the stored ones (a real field's spectrum).
__global__ void k_z_c2r(double2* A, long nlines, int nz, int nzh, double scale) {
    extern __shared__ double2 io_sm[];
    double2* x = io_sm;
    double2* w = io_sm + nz;
    line_twiddles(w, nz, +1.0);
    for (long L = blockIdx.x; L < nlines; L += gridDim.x) {
        __syncthreads();
        for (int k = threadIdx.x; k < nz; k += blockDim.x) {
            const double2 v = k < nzh ? A[L * nzh + k] : A[L * nzh + (nz - k)];
            x[k] = k < nzh ? v : make_double2(v.x, -v.y);
        }
        __syncthreads();
        double* out = (double*)(A + L * nzh);
        for (int p = threadIdx.x; p < nz; p += blockDim.x) out[p] = scale * line_dft_at(x, w, nz, p).x;
    }
}

static int io_grid(long nlines) { return (int)std::min<long>(nlines, 148L * 16); }

// Forward or inverse in-place DFTs along x and y of the [F][nx][ny][nzh] array A.
static void xy_dft(spk_ctx* c, double2* A, double sign) {
    const long nzh = c->nzh, ny = c->ny, nx = c->nx;
    const long nc = (long)c->nc;
    const long lx = (long)c->F * ny * nzh, ly = (long)c->F * nx * nzh;
    // x lines: (f, j, k), elements ny*nzh apart
    k_line_dft<<<io_grid(lx), 256, sizeof(double2) * 2 * nx, c->stream>>>(A, lx, (int)nx, ny * nzh, ny * nzh, nc, 1, 1,
                                                                          0, sign);
    // y lines: (f, i, k), elements nzh apart
    k_line_dft<<<io_grid(ly), 256, sizeof(double2) * 2 * ny, c->stream>>>(A, ly, (int)ny, nzh, nx * nzh, nc, nzh,
                                                                          ny * nzh, 1, sign);
    c->launches += 2;
}

// UnshearComplexVec (cuda_kernels_generic.cu:425-439): every mode times
// exp(-i ky prefactor / 2), a translation along y
__global__ void k_unshear(DevGrid g, double2* X, int F, double prefactor) {
    const size_t n = g.nc * (size_t)F;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const size_t gi = q % g.nc;
        const int j = (int)((gi / g.nzh) % g.ny);
        const double ky = g.ky[j];
        const double cr = cos(-0.5 * ky * prefactor), ci = sin(-0.5 * ky * prefactor);
        const double2 v = X[q];
        X[q] = make_double2(v.x * cr - v.y * ci, v.x * ci + v.y * cr);
    }
}

// The real fields of the state into R (host or device); with the shearing
// box and unshear set, first InputOutput::UnshearOutput's translation at
// time t (unshear_output.cu: tvelocity = fmod(t, 2 Ly / (S Lx)), prefactor
// tvelocity Lx S), as the snapshots hold them.
static int state_real_out(spk_ctx* c, double* R, int where, bool unshear, double t) {
    if (!c || !R) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_get_state_real acts on single-box contexts");
    const long lines = (long)c->F * c->nx * c->ny;
    CK(cudaMemcpyAsync(c->S, c->U, sizeof(double2) * c->nc * c->F, cudaMemcpyDeviceToDevice, c->stream));
    if (unshear && c->p.shearing) {
        const spk_params_t& p = c->p;
        const double tvel = fmod(t, 2.0 * p.ly / (p.shear * p.lx));
        k_unshear<<<io_grid((long)(c->nc * c->F / 256 + 1)), 256, 0, c->stream>>>(c->g, c->S, c->F,
                                                                                    tvel * p.lx * p.shear);
        c->launches++;
    }
    xy_dft(c, c->S, +1.0);
    k_z_c2r<<<io_grid(lines), 128, sizeof(double2) * 2 * c->nz, c->stream>>>(
        c->S, lines, c->nz, c->nzh, 1.0 / ((double)c->nx * c->ny * c->nz));
    c->launches++;
    int rc = launch_status(c);
    if (rc) return rc;
    CK(cudaMemcpy2DAsync(R, sizeof(double) * c->nz, c->S, sizeof(double2) * c->nzh, sizeof(double) * c->nz, lines,
                         where ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c->stream));
    if (where) CK(cudaStreamSynchronize(c->stream));
    return SPK_OK;
}

extern "C" int spk_get_state_real(spk_ctx* c, double* R, int where) { return state_real_out(c, R, where, false, 0.0); }

extern "C" int spk_set_state_real(spk_ctx* c, const double* R, int where) {
    if (!c || !R) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_set_state_real acts on single-box contexts");
    const long lines = (long)c->F * c->nx * c->ny;
    double* stage = (double*)c->S;   // F*nx*ny*nz doubles fit in S (F*nc complex)
    CK(cudaMemcpyAsync(stage, R, sizeof(double) * c->nr * c->F, where ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                       c->stream));
    k_z_r2c<<<io_grid(lines), 128, sizeof(double2) * 2 * c->nz, c->stream>>>(stage, c->U, lines, c->nz, c->nzh);
    c->launches++;
    xy_dft(c, c->U, -1.0);
    int rc = launch_status(c);
    if (rc) return rc;
    if (where) CK(cudaStreamSynchronize(c->stream));
    c->dirty = true;
    return SPK_OK;
}

// ---------------------------------------------------------------------------
// HDF5 files
// ---------------------------------------------------------------------------
#include "spk_hdf5.hpp"

static const char* var_name(const spk_ctx* c, int f) {
    if (c->p.heat_equation) return "th";
    static const char* names[7] = {"vx", "vy", "vz", "bx", "by", "bz", "th"};
    if (!c->p.mhd && f == c->TH && c->p.boussinesq) return "th";
    return names[f];
}

extern "C" int spk_h5_write(const char* path, const spk_h5_dataset_t* ds, int nds) {
    if (!path || (nds > 0 && !ds) || nds < 0) return fail(nullptr, SPK_ERR_ARG, "spk_h5_write: bad argument");
    std::vector<spkh5::Dataset> v(nds);
    for (int i = 0; i < nds; i++) {
        if (!ds[i].name || (!ds[i].data && ds[i].n) || (ds[i].type != SPK_H5_F64 && ds[i].type != SPK_H5_I32))
            return fail(nullptr, SPK_ERR_ARG, "spk_h5_write: bad dataset description");
        v[i].name = ds[i].name;
        if (ds[i].type == SPK_H5_F64) {
            v[i].type = spkh5::F64;
            v[i].f64.assign((const double*)ds[i].data, (const double*)ds[i].data + ds[i].n);
        } else {
            v[i].type = spkh5::I32;
            v[i].i32.assign((const int32_t*)ds[i].data, (const int32_t*)ds[i].data + ds[i].n);
        }
    }
    std::string why;
    if (!spkh5::write_file(path, v, &why)) return fail(nullptr, SPK_ERR_ARG, "spk_h5_write: " + why);
    return SPK_OK;
}

extern "C" int spk_h5_read(const char* path, spk_h5_dataset_t* ds, int nds) {
    if (!path || (nds > 0 && !ds) || nds < 0) return fail(nullptr, SPK_ERR_ARG, "spk_h5_read: bad argument");
    spkh5::Reader r;
    std::string why;
    if (!r.open(path, &why)) return fail(nullptr, SPK_ERR_ARG, "spk_h5_read: " + why);
    for (int i = 0; i < nds; i++) {
        spkh5::Dataset d;
        if (!ds[i].name || !ds[i].data || (ds[i].type != SPK_H5_F64 && ds[i].type != SPK_H5_I32))
            return fail(nullptr, SPK_ERR_ARG, "spk_h5_read: bad dataset description");
        if (!r.read(ds[i].name, ds[i].type == SPK_H5_F64 ? spkh5::F64 : spkh5::I32, &d, &why))
            return fail(nullptr, SPK_ERR_ARG, "spk_h5_read: " + why);
        if (d.size() != ds[i].n)
            return fail(nullptr, SPK_ERR_ARG, "spk_h5_read: dataset " + std::string(ds[i].name) + " has " +
                                                  std::to_string(d.size()) + " elements, expected " +
                                                  std::to_string(ds[i].n));
        if (ds[i].type == SPK_H5_F64) memcpy(ds[i].data, d.f64.data(), sizeof(double) * d.f64.size());
        else memcpy(ds[i].data, d.i32.data(), sizeof(int32_t) * d.i32.size());
    }
    return SPK_OK;
}

extern "C" int spk_write_snapshot(spk_ctx* c, const char* path, double t_start, double t_lastsnap, double t_lastvar) {
    if (!c || !path) return SPK_ERR_ARG;
    int rc = pull_scalars(c);
    if (rc) return rc;
    const double t_save = c->h_sc->t;
    const int32_t step = c->h_sc->step;
    std::vector<double> R((size_t)c->F * c->nr);
    rc = state_real_out(c, R.data(), 1, true, t_save);
    if (rc) return rc;
    std::vector<spk_h5_dataset_t> ds;
    ds.push_back({"t_start", SPK_H5_F64, 1, &t_start});
    ds.push_back({"t_save", SPK_H5_F64, 1, (void*)&t_save});
    ds.push_back({"t_lastsnap", SPK_H5_F64, 1, &t_lastsnap});
    ds.push_back({"t_lastvar", SPK_H5_F64, 1, &t_lastvar});
    ds.push_back({"step", SPK_H5_I32, 1, (void*)&step});
    for (int f = 0; f < c->F; f++) ds.push_back({var_name(c, f), SPK_H5_F64, c->nr, R.data() + (size_t)f * c->nr});
    rc = spk_h5_write(path, ds.data(), (int)ds.size());
    if (rc) return fail(c, rc, g_create_error);
    return SPK_OK;
}

extern "C" int spk_read_snapshot(spk_ctx* c, const char* path, double* t_lastsnap, double* t_lastvar) {
    if (!c || !path) return SPK_ERR_ARG;
    double t_save = 0.0, tls = 0.0, tlv = 0.0;
    int32_t step = 0;
    std::vector<double> R((size_t)c->F * c->nr);
    std::vector<spk_h5_dataset_t> ds;
    ds.push_back({"t_save", SPK_H5_F64, 1, &t_save});
    ds.push_back({"t_lastsnap", SPK_H5_F64, 1, &tls});
    ds.push_back({"t_lastvar", SPK_H5_F64, 1, &tlv});
    ds.push_back({"step", SPK_H5_I32, 1, &step});
    for (int f = 0; f < c->F; f++) ds.push_back({var_name(c, f), SPK_H5_F64, c->nr, R.data() + (size_t)f * c->nr});
    int rc = spk_h5_read(path, ds.data(), (int)ds.size());
    if (rc) return fail(c, rc, g_create_error);
    rc = spk_set_state_real(c, R.data(), 1);
    if (rc) return rc;
    rc = spk_set_time(c, t_save, step, tls);
    if (rc) return rc;
    if (t_lastsnap) *t_lastsnap = tls;
    if (t_lastvar) *t_lastvar = tlv;
    return SPK_OK;
}

// ---------------------------------------------------------------------------
// Time-series diagnostics (src/io/spooky_output_timevar.cu:18-213,
// src/io/spooky_output_functions.cu:23-395) as FP64 reductions on the device.
// ---------------------------------------------------------------------------
// Quadratic quantities by Parseval over the half spectrum.  Energy-like sums
// (computeEnergy: weight 2 for every kz index > 0, the Nyquist plane included)
// and correlations (twoFieldCorrelation: the exact grid mean, weight 1 at
// kz = 0 and at the Nyquist plane) are kept apart.  Sums:
//  0 sum_w |k x u|^2        (enstrophy of u, Curl: i k x u)
//  1 sum_p Re(A_u* . u)     (computeHelicity: A = i k x V / k^2, Helicity kernel)
//  2 sum_w |k x B|^2
//  3 sum_p Re(A_B* . B)
//  4 sum_p Re(u* . B)       (cross helicity)
//  5 sum_w k^2 |th|^2       (computeDissipation: Gradient i k th)
//  6 sum_p Re((i k x u)* . (i k th))   (potential vorticity)
__global__ void k_quadratics(DevGrid g, const double2* U, int VEL, int MAG, int TH, int have_u, int have_b,
                             int have_th, double* sums) {
    const size_t nc = g.nc;
    const int nzl = (g.nz % 2 == 0) ? g.nz / 2 : -1;
    const double shx = grid_shx(g);
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % g.nzh);
        const size_t r = gi / g.nzh;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        const double kx = g.kx[i] + shx * g.ky[j], ky = g.ky[j], kz = g.kz[k];
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
        const double we = k > 0 ? 2.0 : 1.0;
        const double wp = (k > 0 && k != nzl) ? 2.0 : 1.0;
        double2 ucx = {0, 0}, ucy = {0, 0}, ucz = {0, 0}, u0 = {0, 0}, u1 = {0, 0}, u2 = {0, 0};
        if (have_u) {
            u0 = U[(size_t)VEL * nc + gi]; u1 = U[(size_t)(VEL + 1) * nc + gi]; u2 = U[(size_t)(VEL + 2) * nc + gi];
            // k x u (real and imaginary parts separately)
            ucx = make_double2(ky * u2.x - kz * u1.x, ky * u2.y - kz * u1.y);
            ucy = make_double2(kz * u0.x - kx * u2.x, kz * u0.y - kx * u2.y);
            ucz = make_double2(kx * u1.x - ky * u0.x, kx * u1.y - ky * u0.y);
            s[0] += we * (ucx.x * ucx.x + ucx.y * ucx.y + ucy.x * ucy.x + ucy.y * ucy.y + ucz.x * ucz.x + ucz.y * ucz.y);
            // A = i (k x u) / k^2: Re(A* . u) = Re(-i conj(k x u) . u) / k^2 = Im(conj(k x u) . u) / k^2
            const double im = (ucx.x * u0.y - ucx.y * u0.x) + (ucy.x * u1.y - ucy.y * u1.x) + (ucz.x * u2.y - ucz.y * u2.x);
            s[1] += wp * ik2 * im;
        }
        if (have_b) {
            const double2 b0 = U[(size_t)MAG * nc + gi], b1 = U[(size_t)(MAG + 1) * nc + gi], b2 = U[(size_t)(MAG + 2) * nc + gi];
            const double2 cx = make_double2(ky * b2.x - kz * b1.x, ky * b2.y - kz * b1.y);
            const double2 cy = make_double2(kz * b0.x - kx * b2.x, kz * b0.y - kx * b2.y);
            const double2 cz = make_double2(kx * b1.x - ky * b0.x, kx * b1.y - ky * b0.y);
            s[2] += we * (cx.x * cx.x + cx.y * cx.y + cy.x * cy.x + cy.y * cy.y + cz.x * cz.x + cz.y * cz.y);
            const double im = (cx.x * b0.y - cx.y * b0.x) + (cy.x * b1.y - cy.y * b1.x) + (cz.x * b2.y - cz.y * b2.x);
            s[3] += wp * ik2 * im;
            if (have_u)
                s[4] += wp * (u0.x * b0.x + u0.y * b0.y + u1.x * b1.x + u1.y * b1.y + u2.x * b2.x + u2.y * b2.y);
        }
        if (have_th) {
            const double2 t = U[(size_t)TH * nc + gi];
            s[5] += we * k2 * (t.x * t.x + t.y * t.y);
            if (have_u) {
                // (i k x u)* . (i k th) = conj(k x u) . k th
                const double2 d = make_double2(ucx.x * kx + ucy.x * ky + ucz.x * kz, ucx.y * kx + ucy.y * ky + ucz.y * kz);
                s[6] += wp * (d.x * t.x + d.y * t.y);
            }
        }
    }
    for (int q = 0; q < 7; q++) {
        double v = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sums[q], v);
    }
}

// Pointwise means over the real magnetic field (padded rows of 2*nzh
// doubles per (i, j), as the C2R above leaves them):
//  7 |B_z| / (1e-16 + |B|)          averagebz (bUnitvector + DoubleAbsolute)
//  8 (B_z / (1e-16 + |B|))^2        averagebz2
//  9 acosf(|B_x| / (1e-16 + |B_h|))  averagephiB (AngleHorizPlane, single-precision acos)
// (user_defined_cuda_kernels.cu:17-46)
__global__ void k_bstats(const double* R, size_t field_stride, long lines, int nz, int nzh, double* sums) {
    double s[3] = {0, 0, 0};
    const long n = lines * nz;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
        const long L = q / nz;
        const int p = (int)(q - L * nz);
        const size_t at = (size_t)L * 2 * nzh + p;
        const double bx = R[at], by = R[field_stride + at], bz = R[2 * field_stride + at];
        const double nb = 1e-16 + sqrt(bx * bx + by * by + bz * bz);
        const double uz = bz / nb;
        s[0] += fabs(uz);
        s[1] += uz * uz;
        const double nh = 1e-16 + sqrt(bx * bx + by * by);
        s[2] += (double)acosf((float)(fabs(bx) / nh));
    }
    for (int q = 0; q < 3; q++) {
        double v = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sums[7 + q], v);
    }
}

extern "C" int spk_diagnostics(spk_ctx* c, spk_diagnostics_t* out) {
    if (!c || !out) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_diagnostics acts on single-box contexts");
    const bool hu = c->p.incompressible, hb = c->p.incompressible && c->p.mhd;
    const bool ht = c->p.heat_equation || c->p.boussinesq;
    CK(cudaMemsetAsync(c->d_sums, 0, sizeof(double) * 16, c->stream));
    k_quadratics<<<ew_blocks(c->nc), 256, 0, c->stream>>>(c->g, c->U, c->VEL, c->MAG, c->TH, hu, hb, ht, c->d_sums);
    c->launches++;
    if (hb) {
        const long lines = (long)c->F * c->nx * c->ny;
        CK(cudaMemcpyAsync(c->S, c->U, sizeof(double2) * c->nc * c->F, cudaMemcpyDeviceToDevice, c->stream));
        xy_dft(c, c->S, +1.0);
        k_z_c2r<<<io_grid(lines), 128, sizeof(double2) * 2 * c->nz, c->stream>>>(
            c->S, lines, c->nz, c->nzh, 1.0 / ((double)c->nx * c->ny * c->nz));
        const double* R = (const double*)(c->S + (size_t)c->MAG * c->nc);
        k_bstats<<<ew_blocks(c->nr), 256, 0, c->stream>>>(R, 2 * c->nc, (long)c->nx * c->ny, c->nz, c->nzh, c->d_sums);
        c->launches += 2;
    }
    int rc = launch_status(c);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->h_sums, c->d_sums, sizeof(double) * 16, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double n = (double)c->nx * c->ny * c->nz, n2 = n * n;
    const double* s = c->h_sums;
    out->w2 = hu ? 0.5 * s[0] / n2 : -1.0;
    out->hv = hu ? s[1] / n2 : -1.0;
    out->j2 = hb ? 0.5 * s[2] / n2 : -1.0;
    out->hm = hb ? s[3] / n2 : -1.0;
    out->hc = hb ? s[4] / n2 : -1.0;
    out->thetaB = hb ? s[7] / n : -1.0;
    out->bz2 = hb ? s[8] / n : -1.0;
    out->phiB = hb ? s[9] / n : -1.0;
    // with anisotropic conduction and MHD the reference reports the field-aligned
    // dissipation instead (computeAnisoDissipation), which is not computed here
    out->dissgradT = (ht && !(c->p.anisotropic_diffusion && c->p.mhd)) ? 0.5 * s[5] / n2 : -1.0;
    out->pv = (ht && hu) ? s[6] / n2 : -1.0;
    return SPK_OK;
}
