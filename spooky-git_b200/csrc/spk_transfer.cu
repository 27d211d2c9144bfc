// spk_transfer.cu -- transfer spectra of InputOutput::WriteSpectrumOutput
// (src/io/spooky_output_spectrum.cu:186-460) and the field-aligned conduction
// terms of the time series (spooky_output_functions.cu:257-335), on the
// library's passes (included by spk_api.cu).
//
// Each term is built the way the reference builds it -- real-space products,
// their R2C, a masked wavenumber contraction -- on the pass buffers: the x
// and y inverse passes of the needed fields, the z pass forming the products
// (ShearMatrix for the advection terms, MagneticEmf, EnergyFluxVector, the
// anisotropic flux with chi = 1), the y and x forward passes, and a
// contraction kernel writing the term into the RK scratch S (free between
// steps).  The shell spectrum of (field, term) is the one of spk_spectrum.

enum TransferKind { TR_ADVEC, TR_EMF, TR_LORENTZ, TR_THADV, TR_HEL, TR_ANISO_DISS, TR_ANISO_INJ };

struct TermArgs {
    DevGrid g;
    const void* P;          // product channels after the x-forward pass (pass type, kept modes)
    size_t cs;              // channel stride of P (elements)
    const double2* V;       // state field(s) for the helicity term
    double2* T;             // term [3][nc] (or [1][nc])
    int kind, part;         // part: 1 first, 2 second half of the shear matrix (advection)
};

// One mode of the term: NonLinAdvection (cuda_kernels.cu:101-123, the
// symmetric matrix in two halves, the second one added), MagneticShear
// (:257-272), NonLinBoussinesqAdv (:293-304), DivergenceMask
// (cuda_kernels_generic.cu:315-334), Helicity (:474-510: i k x V / k^2).
// Modes outside the 2/3 mask are 0 (their product spectra were not formed).
template <typename T>
__global__ void k_term(const __grid_constant__ TermArgs a) {
    const size_t nc = a.g.nc;
    const double shx = grid_shx(a.g);
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc; gi += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(gi % a.g.nzh);
        const size_t r = gi / a.g.nzh;
        const int j = (int)(r % a.g.ny), i = (int)(r / a.g.ny);
        const double kx = a.g.kx[i] + shx * a.g.ky[j], ky = a.g.ky[j], kz = a.g.kz[k];
        if (a.kind == TR_HEL) {
            const double k2 = kx * kx + ky * ky + kz * kz;
            const double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
            const double2 v0 = a.V[gi], v1 = a.V[nc + gi], v2 = a.V[2 * nc + gi];
            // (k x V): real and imaginary parts; i (k x V) / k^2
            const double2 c0 = d2(ky * v2.x - kz * v1.x, ky * v2.y - kz * v1.y);
            const double2 c1 = d2(kz * v0.x - kx * v2.x, kz * v0.y - kx * v2.y);
            const double2 c2 = d2(kx * v1.x - ky * v0.x, kx * v1.y - ky * v0.y);
            a.T[gi] = d2(-ik2 * c0.y, ik2 * c0.x);
            a.T[nc + gi] = d2(-ik2 * c1.y, ik2 * c1.x);
            a.T[2 * nc + gi] = d2(-ik2 * c2.y, ik2 * c2.x);
            continue;
        }
        const double m = a.g.mx[i] * a.g.my[j] * a.g.mz[k];
        const int nt = (a.kind == TR_THADV || a.kind == TR_ANISO_DISS || a.kind == TR_ANISO_INJ) ? 1 : 3;
        double2 out[3] = {d2(0.0, 0.0), d2(0.0, 0.0), d2(0.0, 0.0)};
        if (m != 0.0) {
            const size_t pi = ((size_t)i * a.g.ny + j) * a.g.nzs + k;
            const C2<T>* P = (const C2<T>*)a.P;
            double2 p[3];
            for (int q = 0; q < 3; q++) {
                const C2<T> v = P[(size_t)q * a.cs + pi];
                p[q] = d2((double)v.x, (double)v.y);
            }
            // s = the contraction (complex); the term is -i m s or i m s
            double2 s[3];
            double sign = -1.0;   // -i
            if (a.kind == TR_ADVEC || a.kind == TR_LORENTZ) {
                if (a.part == 1) {   // S_xx S_xy S_xz
                    s[0] = d2(kx * p[0].x + ky * p[1].x + kz * p[2].x, kx * p[0].y + ky * p[1].y + kz * p[2].y);
                    s[1] = d2(kx * p[1].x, kx * p[1].y);
                    s[2] = d2(kx * p[2].x, kx * p[2].y);
                } else {             // S_yy S_yz S_zz
                    s[0] = d2(0.0, 0.0);
                    s[1] = d2(ky * p[0].x + kz * p[1].x, ky * p[0].y + kz * p[1].y);
                    s[2] = d2(ky * p[1].x + kz * p[2].x, ky * p[1].y + kz * p[2].y);
                }
            } else if (a.kind == TR_EMF) {   // i m (k x E)
                sign = 1.0;
                s[0] = d2(ky * p[2].x - kz * p[1].x, ky * p[2].y - kz * p[1].y);
                s[1] = d2(kz * p[0].x - kx * p[2].x, kz * p[0].y - kx * p[2].y);
                s[2] = d2(kx * p[1].x - ky * p[0].x, kx * p[1].y - ky * p[0].y);
            } else {                       // -i m k.F (advection of theta); i m k.q (divergence)
                sign = a.kind == TR_THADV ? -1.0 : 1.0;
                s[0] = d2(kx * p[0].x + ky * p[1].x + kz * p[2].x, kx * p[0].y + ky * p[1].y + kz * p[2].y);
            }
            for (int q = 0; q < nt; q++) out[q] = d2(-sign * m * s[q].y, sign * m * s[q].x);
        }
        for (int q = 0; q < nt; q++) {
            if ((a.kind == TR_ADVEC || a.kind == TR_LORENTZ) && a.part == 2) {
                const double2 o = a.T[q * nc + gi];
                a.T[q * nc + gi] = d2(o.x + out[q].x, o.y + out[q].y);
            } else {
                a.T[q * nc + gi] = out[q];
            }
        }
    }
}

static int transfer_kind(const std::string& name, int* kind) {
    static const char* names[] = {"advec", "emfpower", "lorentz", "th_advec", "helicity", "th_aniso_diss", "th_aniso_inj"};
    for (int i = 0; i < 7; i++)
        if (name == names[i]) { *kind = i; return SPK_OK; }
    return SPK_ERR_ARG;
}

// x and y inverse passes of nch state fields from `first` into bufB channels c0..
static void inverse_fields(spk_ctx* c, int first, int nch, int c0) {
    AxisArgs a = axis_args(c, 0);
    a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
    add_job(c, a, c->U + (size_t)first * c->nc, chan(c, c->bufA, c0), nch, 1, 0, 0);
    axis(c, a, +1);
    AxisArgs b = axis_args(c, 1);
    add_job(c, b, chan(c, c->bufA, c0), chan(c, c->bufB, c0), nch, 0, 0, 0);
    axis(c, b, +1);
}

static void forward_products(spk_ctx* c, int nch) {
    pass_y_forward(c, nch, c->bufA, c->bufB);
    AxisArgs f = axis_args(c, 0);
    f.kcols = c->kz_keep;
    f.row_filter = 1;
    f.outer_filter = 1;
    add_job(c, f, c->bufB, c->bufA, nch, 0, 0, 0);
    if (f.kcols > 0) axis(c, f, -1);
}

static void launch_term(spk_ctx* c, TermArgs& t) {
    t.g = c->g;
    t.P = c->bufA;
    t.cs = c->g.ncs;
    t.T = c->S;
    c->launches++;
    if (c->fp32) k_term<float><<<ew_blocks(c->nc), 256, 0, c->stream>>>(t);
    else k_term<double><<<ew_blocks(c->nc), 256, 0, c->stream>>>(t);
}

// The term of `kind` into S ([3][nc], or [1][nc] for the scalar terms).
static int transfer_term(spk_ctx* c, int kind) {
    const bool mhd = c->p.mhd, bous = c->p.boussinesq, aniso = c->p.anisotropic_diffusion;
    if (!c->p.incompressible) return fail(c, SPK_ERR_UNSUPPORTED, "transfer spectra need the incompressible module");
    if ((kind == TR_EMF || kind == TR_LORENTZ || kind == TR_HEL) && !mhd)
        return fail(c, SPK_ERR_UNSUPPORTED, "this transfer spectrum needs the MHD module");
    if (kind == TR_THADV && !bous) return fail(c, SPK_ERR_UNSUPPORTED, "th_advec needs the Boussinesq module");
    if ((kind == TR_ANISO_DISS || kind == TR_ANISO_INJ) && !(aniso && mhd && bous))
        return fail(c, SPK_ERR_UNSUPPORTED, "the anisotropic conduction terms need MHD, Boussinesq and anisotropic conduction");
    TermArgs t;
    memset(&t, 0, sizeof(t));
    t.kind = kind;
    if (kind == TR_HEL) {
        t.V = c->U + (size_t)c->MAG * c->nc;
        launch_term(c, t);
        return launch_status(c);
    }
    if (kind == TR_ADVEC || kind == TR_LORENTZ) {
        // the symmetric matrix in two halves of three channels (an HD
        // context's buffers hold five)
        const int base = kind == TR_ADVEC ? c->VEL : c->MAG;
        for (int part = 1; part <= 2; part++) {
            inverse_fields(c, base, 3, 0);
            ZArgs z = z_args(c);
            z.mode = ZM_PRODUCTS;
            z.nin = 3; z.ch_u = 0;
            z.shear_part = part;
            z.nout = 3;
            zpass(c, z);
            forward_products(c, 3);
            t.part = part;
            launch_term(c, t);
        }
        return launch_status(c);
    }
    ZArgs z = z_args(c);
    z.mode = ZM_PRODUCTS;
    z.nout = 3;
    if (kind == TR_EMF) {
        inverse_fields(c, c->VEL, 6, 0);   // u (0-2), B (3-5)
        z.nin = 6; z.ch_u = 0; z.ch_b = 3; z.mhd = 1;
    } else if (kind == TR_THADV) {
        inverse_fields(c, c->VEL, 3, 0);
        AxisArgs a = axis_args(c, 0);
        a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
        add_job(c, a, c->U + (size_t)c->TH * c->nc, chan(c, c->bufA, 3), 1, 1, 0, 0);
        axis(c, a, +1);
        AxisArgs b = axis_args(c, 1);
        add_job(c, b, chan(c, c->bufA, 3), chan(c, c->bufB, 3), 1, 0, 0, 0);
        axis(c, b, +1);
        z.nin = 4; z.ch_u = 0; z.ch_th = 3; z.bous = 1;
    } else {
        // B (0-2), theta (3), d/dx theta (4), d/dy theta (5), d/dz theta derived in the z pass
        AxisArgs a = axis_args(c, 0);
        a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
        add_job(c, a, c->U + (size_t)c->MAG * c->nc, chan(c, c->bufA, 0), 3, 1, 0, 0);
        add_job(c, a, c->U + (size_t)c->TH * c->nc, chan(c, c->bufA, 3), 1, 1, 0, 0);
        add_job(c, a, c->U + (size_t)c->TH * c->nc, chan(c, c->bufA, 4), 1, 1, 1, 0);
        axis(c, a, +1);
        AxisArgs b = axis_args(c, 1);
        add_job(c, b, c->bufA, c->bufB, 5, 0, 0, 0);
        add_job(c, b, chan(c, c->bufA, 3), chan(c, c->bufB, 5), 1, 0, 1, 0);
        axis(c, b, +1);
        z.ch_b = 0; z.aniso = 1; z.chi = 1.0;
        if (kind == TR_ANISO_DISS) {
            // ComputeAnisotropicHeatFlux with omega_T^2 = 0 and chi = 1 (anisotropic_conduction.cu:107-160)
            z.nin = 6; z.ch_th = 3; z.ch_gx = 4; z.ch_gy = 5; z.derive_gz = 1; z.omegaT2 = 0.0;
        } else {
            // Computebbstrat: b b_s / |b|^2 (anisotropic_conduction.cu:69-104)
            z.nin = 3; z.omegaT2 = 1.0;
        }
    }
    zpass(c, z);
    forward_products(c, 3);
    launch_term(c, t);
    return launch_status(c);
}

extern "C" int spk_transfer_spectra(spk_ctx* c, const char* kind_name, double* out, int max_bins, int* ncomp,
                                    int* nbins, double* deltak, double* totals) {
    if (!c || !kind_name) return SPK_ERR_ARG;
    if (c->nb != 1) return fail(c, SPK_ERR_UNSUPPORTED, "spk_transfer_spectra acts on single-box contexts");
    int kind = 0;
    if (transfer_kind(kind_name, &kind)) return fail(c, SPK_ERR_ARG, std::string("unknown transfer spectrum ") + kind_name);
    if (c->nbins < 1) return fail(c, SPK_ERR_UNSUPPORTED, "no spectral bins for this grid");
    int rc = transfer_term(c, kind);
    if (rc) return rc;
    // the field each component pairs with: u (advection, Lorentz), B (EMF, helicity), theta
    int f0 = c->VEL, nt = 3;
    if (kind == TR_EMF || kind == TR_HEL) f0 = c->MAG;
    if (kind == TR_THADV || kind == TR_ANISO_DISS || kind == TR_ANISO_INJ) { f0 = c->TH; nt = 1; }
    if (ncomp) *ncomp = nt;
    if (nbins) *nbins = c->nbins;
    if (deltak) *deltak = c->deltak;
    const double inv_n = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
    const int grid = (int)std::min<size_t>((c->nc + 255) / 256, (size_t)c->num_sms * 8);
    std::vector<double> h((size_t)c->nbins + 1);
    for (int q = 0; q < nt; q++) {
        CK(cudaMemsetAsync(c->d_spec, 0, sizeof(double) * (size_t)(c->nbins + 1), c->stream));
        k_spectrum<<<grid, 256, sizeof(double) * (size_t)c->nbins, c->stream>>>(
            c->g, c->U + (size_t)(f0 + q) * c->nc, c->S + (size_t)q * c->nc, c->nbins, c->deltak, inv_n, c->d_spec);
        c->launches++;
        rc = launch_status(c);
        if (rc) return rc;
        CK(cudaMemcpyAsync(h.data(), c->d_spec, sizeof(double) * (size_t)(c->nbins + 1), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (out) for (int m = 0; m < std::min(max_bins, c->nbins); m++) out[(size_t)q * max_bins + m] = h[(size_t)m];
        if (totals) totals[q] = h[(size_t)c->nbins];
    }
    return SPK_OK;
}
