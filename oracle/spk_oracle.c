/*
 * spk_oracle.c -- CPU FP64 restatement of the SPOOKY hot path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); never on
 * the product path.  Compiled with -ffp-contract=off so that the wavevector
 * and mask expressions round exactly as the reference's host code does.
 *
 * Reference = LorenzoLMP/spooky-git; citations are file:line in that tree.
 */
#include "spk_oracle.h"
#include "spk_closure.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cpx;

static inline cpx c_add(cpx a, cpx b) { cpx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cpx c_sub(cpx a, cpx b) { cpx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cpx c_mul(cpx a, cpx b) { cpx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cpx c_conj(cpx a) { cpx r = {a.re, -a.im}; return r; }
static inline cpx c_scale(double s, cpx a) { cpx r = {s * a.re, s * a.im}; return r; }
/* i * a */
static inline cpx c_muli(cpx a) { cpx r = {-a.im, a.re}; return r; }

/* ======================================================================
 * FFT: mixed-radix Stockham (decimation in frequency), written from the
 * DFT definition  X[k] = sum_n x[n] exp(sign * 2 pi i n k / N).
 * Stage with radix R on current length n (stride s = N/n, m = n/R):
 *   a_r = x[q + s(p + r m)],  y[q + s(R p + t)] = w_n^{p t} sum_r a_r w_R^{r t}
 * ====================================================================== */
#define PI_L 3.141592653589793238462643383279502884L

typedef struct {
    int n, nst;
    int radix[40];
    cpx* tw;   /* tw[k] = exp(-2 pi i k / n) */
} fftplan;

static void plan_init(fftplan* p, int n) {
    p->n = n;
    p->nst = 0;
    int r = n;
    while (r % 4 == 0) { p->radix[p->nst++] = 4; r /= 4; }
    while (r % 2 == 0) { p->radix[p->nst++] = 2; r /= 2; }
    while (r % 3 == 0) { p->radix[p->nst++] = 3; r /= 3; }
    while (r % 5 == 0) { p->radix[p->nst++] = 5; r /= 5; }
    for (int f = 7; r > 1; f += 2) {
        while (r % f == 0) { p->radix[p->nst++] = f; r /= f; }
    }
    p->tw = (cpx*)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; k++) {
        long double a = 2.0L * PI_L * (long double)k / (long double)n;
        p->tw[k].re = (double)cosl(a);
        p->tw[k].im = -(double)sinl(a);
    }
}

static void plan_free(fftplan* p) { free(p->tw); p->tw = NULL; }

/* x, y: n*vl complex, element (idx, v) at [idx*vl + v].  Result in x. */
static void fft_vec(const fftplan* p, cpx* x, cpx* y, int vl, int sign) {
    const int n = p->n;
    int s = 1;
    cpx* a = x;
    cpx* b = y;
    cpx in[64], out[64];
    for (int st = 0; st < p->nst; st++) {
        const int R = p->radix[st];
        const int ncur = n / s;
        const int m = ncur / R;
        const int wstep = n / R;
        for (int pp = 0; pp < m; pp++) {
            for (int q = 0; q < s; q++) {
                for (int v = 0; v < vl; v++) {
                    for (int r = 0; r < R; r++) in[r] = a[(size_t)(q + s * (pp + r * m)) * vl + v];
                    if (R == 2) {
                        out[0] = c_add(in[0], in[1]);
                        out[1] = c_sub(in[0], in[1]);
                    } else if (R == 4) {
                        cpx s02 = c_add(in[0], in[2]), d02 = c_sub(in[0], in[2]);
                        cpx s13 = c_add(in[1], in[3]), d13 = c_sub(in[1], in[3]);
                        /* forward: w4 = -i ; inverse: w4 = +i */
                        cpx jd13 = c_muli(d13);
                        out[0] = c_add(s02, s13);
                        out[2] = c_sub(s02, s13);
                        if (sign < 0) { out[1] = c_sub(d02, jd13); out[3] = c_add(d02, jd13); }
                        else          { out[1] = c_add(d02, jd13); out[3] = c_sub(d02, jd13); }
                    } else {
                        for (int t = 0; t < R; t++) {
                            cpx acc = {0.0, 0.0};
                            for (int r = 0; r < R; r++) {
                                cpx w = p->tw[(size_t)((r * t) % R) * wstep];
                                if (sign > 0) w = c_conj(w);
                                acc = c_add(acc, c_mul(in[r], w));
                            }
                            out[t] = acc;
                        }
                    }
                    for (int t = 0; t < R; t++) {
                        cpx o = out[t];
                        if (t > 0 && pp > 0) {
                            cpx w = p->tw[(size_t)pp * t * s];
                            if (sign > 0) w = c_conj(w);
                            o = c_mul(o, w);
                        }
                        b[(size_t)(q + s * (R * pp + t)) * vl + v] = o;
                    }
                }
            }
        }
        cpx* tmp = a; a = b; b = tmp;
        s *= R;
    }
    if (a != x) memcpy(x, a, sizeof(cpx) * (size_t)n * vl);
}

void orc_fft1d(int n, const double* in, double* out, int sign) {
    fftplan p;
    plan_init(&p, n);
    cpx* x = (cpx*)malloc(sizeof(cpx) * n);
    cpx* y = (cpx*)malloc(sizeof(cpx) * n);
    memcpy(x, in, sizeof(cpx) * n);
    fft_vec(&p, x, y, 1, sign);
    memcpy(out, x, sizeof(cpx) * n);
    free(x); free(y); plan_free(&p);
}

void orc_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* ======================================================================
 * 3-D transforms on the reference layouts:
 *   complex C[i][j][k], k < NZ/2+1;  real R[i][j][z] (unpadded).
 * c2r follows src/cuda/cufft_routines.cu:59-81: input scaled by 1/(NX NY NZ)
 * (scaleKernel) then Z2D.  Inverse order: x, y, then the z C2R, whose DC and
 * Nyquist imaginary parts are discarded (real-signal convention).
 * r2c (D2Z) is unnormalised: z R2C, then y, then x.
 * ====================================================================== */
typedef struct {
    int nx, ny, nz, nzh;
    size_t nc, nr;
    fftplan px, py, pz;
} grid3;

#define VBLK 8

static void axis_pass(const grid3* g, cpx* a, int axis, int sign) {
    /* axis 0: x (stride ny*nzh), axis 1: y (stride nzh); blocks of VBLK k's */
    const int nzh = g->nzh;
    const int n = axis == 0 ? g->nx : g->ny;
    const int nouter = axis == 0 ? g->ny : g->nx;
    const size_t stride = axis == 0 ? (size_t)g->ny * nzh : (size_t)nzh;
    const fftplan* p = axis == 0 ? &g->px : &g->py;
    const int nkb = (nzh + VBLK - 1) / VBLK;
    #pragma omp parallel
    {
        cpx* bx = (cpx*)malloc(sizeof(cpx) * (size_t)n * VBLK);
        cpx* by = (cpx*)malloc(sizeof(cpx) * (size_t)n * VBLK);
        #pragma omp for schedule(static)
        for (long job = 0; job < (long)nouter * nkb; job++) {
            int o = (int)(job / nkb), kb = (int)(job % nkb);
            int k0 = kb * VBLK, vl = nzh - k0 < VBLK ? nzh - k0 : VBLK;
            size_t base = axis == 0 ? (size_t)o * nzh : (size_t)o * g->ny * nzh;
            for (int t = 0; t < n; t++)
                for (int v = 0; v < vl; v++) bx[(size_t)t * vl + v] = a[base + t * stride + k0 + v];
            fft_vec(p, bx, by, vl, sign);
            for (int t = 0; t < n; t++)
                for (int v = 0; v < vl; v++) a[base + t * stride + k0 + v] = bx[(size_t)t * vl + v];
        }
        free(bx); free(by);
    }
}

static void c2r_3d(const grid3* g, const cpx* in, double* out, cpx* work) {
    const double scale = 1.0 / ((double)g->nx * (double)g->ny * (double)g->nz);
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)g->nc; i++) work[i] = c_scale(scale, in[i]);
    axis_pass(g, work, 0, +1);
    axis_pass(g, work, 1, +1);
    const int nz = g->nz, nzh = g->nzh;
    #pragma omp parallel
    {
        cpx* zx = (cpx*)malloc(sizeof(cpx) * nz);
        cpx* zy = (cpx*)malloc(sizeof(cpx) * nz);
        #pragma omp for schedule(static)
        for (long l = 0; l < (long)g->nx * g->ny; l++) {
            const cpx* L = work + (size_t)l * nzh;
            zx[0].re = L[0].re; zx[0].im = 0.0;
            for (int k = 1; k < nzh; k++) {
                if (2 * k == nz) { zx[k].re = L[k].re; zx[k].im = 0.0; }
                else { zx[k] = L[k]; zx[nz - k] = c_conj(L[k]); }
            }
            fft_vec(&g->pz, zx, zy, 1, +1);
            double* o = out + (size_t)l * nz;
            for (int z = 0; z < nz; z++) o[z] = zx[z].re;
        }
        free(zx); free(zy);
    }
}

static void r2c_3d(const grid3* g, const double* in, cpx* out) {
    const int nz = g->nz, nzh = g->nzh;
    #pragma omp parallel
    {
        cpx* zx = (cpx*)malloc(sizeof(cpx) * nz);
        cpx* zy = (cpx*)malloc(sizeof(cpx) * nz);
        #pragma omp for schedule(static)
        for (long l = 0; l < (long)g->nx * g->ny; l++) {
            const double* r = in + (size_t)l * nz;
            for (int z = 0; z < nz; z++) { zx[z].re = r[z]; zx[z].im = 0.0; }
            fft_vec(&g->pz, zx, zy, 1, -1);
            for (int k = 0; k < nzh; k++) out[(size_t)l * nzh + k] = zx[k];
        }
        free(zx); free(zy);
    }
    axis_pass(g, out, 1, -1);
    axis_pass(g, out, 0, -1);
}

/* ======================================================================
 * Context
 * ====================================================================== */
struct orc_ctx {
    spk_params_t p;
    int F, VX, VY, VZ, BX, BY, BZ, TH, VEL, MAG;
    grid3 g;
    double *kx, *ky, *kz;          /* 1-D wavevector tables (wavevector.cu:66-76) */
    double *mx, *my, *mz;          /* separable 2/3 mask factors (wavevector.cu:82-95) */
    double kxmax, kymax, kzmax, kmax;
    int sts_pos[8], sts_index[8], nsts;
    cpx *U, *dU, *S, *tmp, *work;
    double *realbuf, *rtmp;
    cpx *rdU, *rdU0, *rUc0, *rUc1;
    double t, dt, dt_hyp, dt_par, dt_sts, t_lastsnap;
    int step;
    /* shearing box: the remap clock and the shear of the wavevector in use,
     * kx = kx0 + shx ky with shx = shear * (tremap of the stage) */
    double tremap, shx;
    /* learned closure (spk_closure.c): parameters, Delta^2, the real-space
     * closure terms -2 nu_t S (5) and -eta_t J (3), the gradients A, G (18) */
    int closure_on;
    double cparams[SPK_CLOSURE3_NPARAM];   /* variant 3's count, the larger */
    double delta2, nu_t_max, eta_t_max;
    double *rclos, *rgrad;
    cpx* ctmp;
};

int orc_num_fields(const orc_ctx* c) { return c->F; }
size_t orc_ncomplex(const orc_ctx* c) { return c->g.nc; }

/* Parameters::popVariablesGrid (src/parameters/parameters.cu:568-654) */
static void pop_variables(orc_ctx* c) {
    const spk_params_t* p = &c->p;
    c->F = 0; c->VX = c->VY = c->VZ = c->BX = c->BY = c->BZ = c->TH = c->VEL = c->MAG = 0;
    if (p->heat_equation) { c->TH = 0; c->F = 1; }
    else if (p->incompressible) {
        c->VX = 0; c->VY = 1; c->VZ = 2; c->F = 3; c->VEL = 0;
        if (p->mhd) {
            c->BX = 3; c->BY = 4; c->BZ = 5; c->F += 3; c->MAG = 3;
            if (p->boussinesq) { c->TH = 6; c->F += 1; }
        } else if (p->boussinesq) { c->TH = 3; c->F += 1; }
    }
}

static double shift_time(const spk_params_t* p, double t);

orc_ctx* orc_create(const spk_params_t* p) {
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->p = *p;
    pop_variables(c);
    grid3* g = &c->g;
    g->nx = p->nx; g->ny = p->ny; g->nz = p->nz; g->nzh = p->nz / 2 + 1;
    g->nc = (size_t)g->nx * g->ny * g->nzh;
    g->nr = (size_t)g->nx * g->ny * g->nz;
    plan_init(&g->px, g->nx); plan_init(&g->py, g->ny); plan_init(&g->pz, g->nz);

    /* Wavevector::Wavevector (src/fields/wavevector.cu:50-112): the exact
     * FP64 expressions, evaluated per 1-D index (they depend on one index). */
    c->kx = (double*)malloc(sizeof(double) * g->nx);
    c->ky = (double*)malloc(sizeof(double) * g->ny);
    c->kz = (double*)malloc(sizeof(double) * g->nzh);
    c->mx = (double*)malloc(sizeof(double) * g->nx);
    c->my = (double*)malloc(sizeof(double) * g->ny);
    c->mz = (double*)malloc(sizeof(double) * g->nzh);
    for (int i = 0; i < g->nx; i++)
        c->kx[i] = (2.0 * M_PI) / p->lx * (fmod((double)i + ((double)g->nx / 2), g->nx) - (double)g->nx / 2);
    for (int j = 0; j < g->ny; j++)
        c->ky[j] = (2.0 * M_PI) / p->ly * (fmod((double)j + ((double)g->ny / 2), g->ny) - (double)g->ny / 2);
    for (int k = 0; k < g->nzh; k++)
        c->kz[k] = p->with2d ? 0.0 : (2.0 * M_PI) / p->lz * (double)k;
    c->kxmax = 2.0 * M_PI / p->lx * ((g->nx / 2) - 1);
    c->kymax = 2.0 * M_PI / p->ly * ((g->ny / 2) - 1);
    c->kzmax = 2.0 * M_PI / p->lz * ((g->nz / 2) - 1);
    if (p->with2d) c->kzmax = 0.0;
    for (int i = 0; i < g->nx; i++) c->mx[i] = 1.0;
    for (int j = 0; j < g->ny; j++) c->my[j] = 1.0;
    for (int k = 0; k < g->nzh; k++) c->mz[k] = 1.0;
    if (p->antialiasing) {
        for (int i = 0; i < g->nx; i++) if (fabs(c->kx[i]) > 2.0 / 3.0 * c->kxmax) c->mx[i] = 0.0;
        for (int j = 0; j < g->ny; j++) if (fabs(c->ky[j]) > 2.0 / 3.0 * c->kymax) c->my[j] = 0.0;
        for (int k = 0; k < g->nzh; k++) if (fabs(c->kz[k]) > 2.0 / 3.0 * c->kzmax) c->mz[k] = 0.0;
        c->kxmax = (2.0 / 3.0) * c->kxmax;
        c->kymax = (2.0 / 3.0) * c->kymax;
        c->kzmax = (2.0 / 3.0) * c->kzmax;
    }
    c->kmax = pow(c->kxmax * c->kxmax + c->kymax * c->kymax + c->kzmax * c->kzmax, 0.5);

    /* RKLegendre ctor: sts_variables_pos / _index (src/rkl/rkl.cu:40-58) */
    c->nsts = 0;
    for (int f = 0; f < c->F; f++) {
        c->sts_pos[f] = -1;
        if (p->supertimestepping && (p->sts_vars_mask >> f & 1u)) {
            c->sts_pos[f] = c->nsts;
            c->sts_index[c->nsts++] = f;
        }
    }

    size_t nc = g->nc, nr = g->nr;
    c->U = (cpx*)calloc(nc * c->F, sizeof(cpx));
    c->dU = (cpx*)calloc(nc * c->F, sizeof(cpx));
    c->S = (cpx*)calloc(nc * c->F, sizeof(cpx));
    c->tmp = (cpx*)calloc(nc * 6, sizeof(cpx));
    c->work = (cpx*)calloc(nc, sizeof(cpx));
    c->realbuf = (double*)calloc(nr * c->F, sizeof(double));
    c->rtmp = (double*)calloc(nr * 6, sizeof(double));
    if (c->nsts > 0) {
        c->rdU = (cpx*)calloc(nc * c->nsts, sizeof(cpx));
        c->rdU0 = (cpx*)calloc(nc * c->nsts, sizeof(cpx));
        c->rUc0 = (cpx*)calloc(nc * c->nsts, sizeof(cpx));
        c->rUc1 = (cpx*)calloc(nc * c->nsts, sizeof(cpx));
    }
    c->t = p->t_initial;
    c->t_lastsnap = 0.0;
    c->step = 0;
    c->delta2 = pow(M_PI / c->kxmax * M_PI / c->kymax * M_PI / c->kzmax, 2.0 / 3.0);
    if (p->shearing) {
        c->tremap = shift_time(p, c->t);
        c->shx = p->shear * c->tremap;
    }
    return c;
}

void orc_destroy(orc_ctx* c) {
    if (!c) return;
    plan_free(&c->g.px); plan_free(&c->g.py); plan_free(&c->g.pz);
    free(c->kx); free(c->ky); free(c->kz); free(c->mx); free(c->my); free(c->mz);
    free(c->U); free(c->dU); free(c->S); free(c->tmp); free(c->work);
    free(c->realbuf); free(c->rtmp);
    free(c->rdU); free(c->rdU0); free(c->rUc0); free(c->rUc1);
    free(c->rclos); free(c->rgrad); free(c->ctmp);
    free(c);
}

/* the shearing box's remap clock (0 without the module) */
double orc_get_tremap(const orc_ctx* c) { return c->tremap; }

void orc_set_state(orc_ctx* c, const double* U) { memcpy(c->U, U, sizeof(cpx) * c->g.nc * c->F); }
void orc_get_state(const orc_ctx* c, double* U) { memcpy(U, c->U, sizeof(cpx) * c->g.nc * c->F); }
/* With the shearing module a new time restarts the remap clock from it, as
 * Supervisor::executeMainLoop does before its loop (supervisor.cu:171-175);
 * the same time keeps the clock. */
void orc_set_time(orc_ctx* c, double t, int step, double t_lastsnap) {
    const int restart = t != c->t;
    c->t = t; c->step = step; c->t_lastsnap = t_lastsnap;
    if (c->p.shearing && restart) {
        c->tremap = shift_time(&c->p, t);
        c->shx = c->p.shear * c->tremap;
    }
}
void orc_get_time(const orc_ctx* c, double* t, double* dt, int* step) {
    if (t) *t = c->t;
    if (dt) *dt = c->dt;
    if (step) *step = c->step;
}

void orc_kgrid(const orc_ctx* c, double* kvec, double* mask, double* kmax4) {
    const grid3* g = &c->g;
    for (int i = 0; i < g->nx; i++)
        for (int j = 0; j < g->ny; j++)
            for (int k = 0; k < g->nzh; k++) {
                size_t idx = (size_t)k + g->nzh * ((size_t)j + (size_t)i * g->ny);
                kvec[idx] = c->kx[i] + c->shx * c->ky[j];   /* sheared */
                kvec[g->nc + idx] = c->ky[j];
                kvec[2 * g->nc + idx] = c->kz[k];
                mask[idx] = c->mx[i] * c->my[j] * c->mz[k];
            }
    kmax4[0] = c->kxmax; kmax4[1] = c->kymax; kmax4[2] = c->kzmax; kmax4[3] = c->kmax;
}

/* Loop over all spectral modes with (kx, ky, kz, mask) of the mode. */
#define FOR_MODES(c)                                                               \
    _Pragma("omp parallel for collapse(2) schedule(static)")                       \
    for (int i_ = 0; i_ < (c)->g.nx; i_++)                                         \
        for (int j_ = 0; j_ < (c)->g.ny; j_++)                                     \
            for (int k_ = 0; k_ < (c)->g.nzh; k_++)

/* kx is sheared: ShearWavevector (cuda_kernels_generic.cu:362-384), shx = 0
 * without the shearing module */
#define MODE_VARS(c)                                                               \
    const size_t id = (size_t)k_ + (c)->g.nzh * ((size_t)j_ + (size_t)i_ * (c)->g.ny); \
    const double kx = (c)->kx[i_] + (c)->shx * (c)->ky[j_], ky = (c)->ky[j_], kz = (c)->kz[k_]; \
    const double mask = (c)->mx[i_] * (c)->my[j_] * (c)->mz[k_];                       \
    (void)kx; (void)ky; (void)kz; (void)mask;

/* Supervisor::Complex2RealFields (src/supervisor/supervisor.cu:261-272) */
static void complex2real(orc_ctx* c, const cpx* Uin, double* R, int nf) {
    for (int f = 0; f < nf; f++) c2r_3d(&c->g, Uin + (size_t)f * c->g.nc, R + (size_t)f * c->g.nr, c->work);
}

/* ---- learned closure terms (include/spooky_b200.h, SPK_CLOSURE_*): the
 * spectral gradients of u and B to real space, then per point the features,
 * the MLP and the terms -2 nu_t S, -eta_t J; maxima of nu_t and eta_t. */
/* The gradients A (9) and G (9) of U in real space into c->rgrad; use_hp:
 * of the small scales |k| > k_c/2 only (variant 2), k_c the smallest
 * dealiased cut-off. */
static void closure_grads(orc_ctx* c, const cpx* U, int use_hp) {
    const size_t nr = c->g.nr, nc = c->g.nc;
    const int mhd = c->p.mhd;
    memset(c->rgrad, 0, sizeof(double) * 18 * nr);
    double hp_k2 = 0.0;
    if (use_hp) {
        double kc = c->kxmax;
        if (c->kymax < kc) kc = c->kymax;
        if (c->kzmax < kc) kc = c->kzmax;
        const double f = c->p.closure_kc_frac > 0.0 ? c->p.closure_kc_frac : 0.5;
        hp_k2 = f * f * kc * kc;
    }
    for (int b = 0; b < (mhd ? 2 : 1); b++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const cpx* X = U + (size_t)((b ? c->MAG : c->VEL) + i) * nc;
                FOR_MODES(c) {
                    MODE_VARS(c)
                    const double kj = j == 0 ? kx : (j == 1 ? ky : kz);
                    const int small = !(hp_k2 > 0.0) || kx * kx + ky * ky + kz * kz > hp_k2;
                    c->ctmp[id] = small ? c_scale(kj, c_muli(X[id])) : (cpx){0.0, 0.0};
                }
                c2r_3d(&c->g, c->ctmp, c->rgrad + (size_t)(9 * b + 3 * i + j) * nr, c->work);
            }
}

static void closure_fields(orc_ctx* c, const cpx* U) {
    const size_t nr = c->g.nr;
    const int mhd = c->p.mhd;
    closure_grads(c, U, c->p.closure == 2);
    double numax = 0.0, etamax = 0.0;
    if (c->p.closure == 3) {
        #pragma omp parallel for schedule(static) reduction(max : numax, etamax)
        for (long q = 0; q < (long)nr; q++) {
            double A[9], G[9], tau[5], e[3], nu, eta;
            for (int r = 0; r < 9; r++) { A[r] = c->rgrad[(size_t)r * nr + q]; G[r] = c->rgrad[(size_t)(9 + r) * nr + q]; }
            orc_closure3_terms(c->cparams, c->delta2, A, G, mhd, tau, e, &nu, &eta);
            for (int r = 0; r < 5; r++) c->rclos[(size_t)r * nr + q] = tau[r];
            for (int r = 0; r < 3; r++) c->rclos[(size_t)(5 + r) * nr + q] = e[r];
            if (nu > numax) numax = nu;
            if (eta > etamax) etamax = eta;
        }
        c->nu_t_max = numax;
        c->eta_t_max = etamax;
        return;
    }
    #pragma omp parallel for schedule(static) reduction(max : numax, etamax)
    for (long q = 0; q < (long)nr; q++) {
        double A[9], G[9], f[8], S5[5], J3[3], o[2];
        for (int r = 0; r < 9; r++) { A[r] = c->rgrad[(size_t)r * nr + q]; G[r] = c->rgrad[(size_t)(9 + r) * nr + q]; }
        const double n = orc_closure_features(A, G, f, S5, J3);
        orc_closure_mlp(c->cparams, f, o);
        const double sc = c->delta2 * n;
        const double nu = sc * (o[0] > 30.0 ? o[0] : log1p(exp(o[0])));
        const double eta = sc * (o[1] > 30.0 ? o[1] : log1p(exp(o[1])));
        for (int r = 0; r < 5; r++) c->rclos[(size_t)r * nr + q] = -2.0 * nu * S5[r];
        for (int r = 0; r < 3; r++) c->rclos[(size_t)(5 + r) * nr + q] = mhd ? -eta * J3[r] : 0.0;
        if (nu > numax) numax = nu;
        if (mhd && eta > etamax) etamax = eta;
    }
    c->nu_t_max = numax;
    c->eta_t_max = etamax;
}

int orc_closure_set(orc_ctx* c, const double* params) {
    if (!params) { c->closure_on = 0; return 0; }
    if (!c->p.incompressible || c->p.boussinesq) return 1;
    memcpy(c->cparams, params, sizeof(double) * (c->p.closure == 3 ? SPK_CLOSURE3_NPARAM : SPK_CLOSURE_NPARAM));
    if (!c->rclos) {
        c->rclos = (double*)calloc(c->g.nr * 8, sizeof(double));
        c->rgrad = (double*)calloc(c->g.nr * 18, sizeof(double));
        c->ctmp = (cpx*)calloc(c->g.nc, sizeof(cpx));
    }
    c->closure_on = 1;
    return 0;
}

/* ---- Physics::BasdevantHydro (src/physics/hydro.cu:19-75) -------------- */
static void basdevant_hydro(orc_ctx* c, const double* rb, cpx* dVel) {
    const size_t nr = c->g.nr, nc = c->g.nc;
    const double* u = rb + (size_t)c->VEL * nr;
    const double* B = rb + (size_t)c->MAG * nr;
    double* T = c->rtmp;
    const int mhd = c->p.mhd;
    /* TracelessShearMatrix / ...MHD (src/cuda/cuda_kernels.cu:39-55, 216-234) */
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nr; i++) {
        double ux = u[i], uy = u[nr + i], uz = u[2 * nr + i];
        if (!mhd) {
            T[i] = (2.0 * ux * ux - uy * uy - uz * uz) / 3.0;
            T[nr + i] = ux * uy;
            T[2 * nr + i] = ux * uz;
            T[3 * nr + i] = (-ux * ux + 2.0 * uy * uy - uz * uz) / 3.0;
            T[4 * nr + i] = uy * uz;
        } else {
            double bx = B[i], by = B[nr + i], bz = B[2 * nr + i];
            T[i] = (2.0 * ux * ux - uy * uy - uz * uz - 2.0 * bx * bx + by * by + bz * bz) / 3.0;
            T[nr + i] = ux * uy - bx * by;
            T[2 * nr + i] = ux * uz - bx * bz;
            T[3 * nr + i] = (-ux * ux + 2.0 * uy * uy - uz * uz + bx * bx - 2.0 * by * by + bz * bz) / 3.0;
            T[4 * nr + i] = uy * uz - by * bz;
        }
    }
    if (c->closure_on)
        for (size_t i = 0; i < 5 * nr; i++) T[i] += c->rclos[i];
    for (int n = 0; n < 5; n++) r2c_3d(&c->g, T + (size_t)n * nr, c->tmp + (size_t)n * nc);
    const cpx* S = c->tmp;
    /* NonLinHydroAdv (src/cuda/cuda_kernels.cu:82-98): overwrites dVel */
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx s0 = S[id], s1 = S[nc + id], s2 = S[2 * nc + id], s3 = S[3 * nc + id], s4 = S[4 * nc + id];
        cpx ax = c_add(c_add(c_scale(kx, s0), c_scale(ky, s1)), c_scale(kz, s2));
        cpx ay = c_add(c_add(c_scale(kx, s1), c_scale(ky, s3)), c_scale(kz, s4));
        cpx az = c_sub(c_add(c_scale(kx, s2), c_scale(ky, s4)), c_scale(kz, c_add(s0, s3)));
        dVel[id] = c_scale(-mask, c_muli(ax));
        dVel[nc + id] = c_scale(-mask, c_muli(ay));
        dVel[2 * nc + id] = c_scale(-mask, c_muli(az));
    }
}

/* ---- Physics::CurlEMF (src/physics/mhd.cu:20-62) ----------------------- */
static void curl_emf(orc_ctx* c, const double* rb, cpx* dMag) {
    const size_t nr = c->g.nr, nc = c->g.nc;
    const double* u = rb + (size_t)c->VEL * nr;
    const double* B = rb + (size_t)c->MAG * nr;
    double* E = c->rtmp;
    /* MagneticEmf (src/cuda/cuda_kernels.cu:240-252) */
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nr; i++) {
        double ux = u[i], uy = u[nr + i], uz = u[2 * nr + i];
        double bx = B[i], by = B[nr + i], bz = B[2 * nr + i];
        E[i] = -by * uz + bz * uy;
        E[nr + i] = bx * uz - bz * ux;
        E[2 * nr + i] = -bx * uy + by * ux;
    }
    if (c->closure_on)
        for (size_t i = 0; i < 3 * nr; i++) E[i] += c->rclos[5 * nr + i];
    for (int n = 0; n < 3; n++) r2c_3d(&c->g, E + (size_t)n * nr, c->tmp + (size_t)n * nc);
    const cpx* M = c->tmp;
    /* MagneticShear (src/cuda/cuda_kernels.cu:257-272): overwrites dMag */
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx e0 = M[id], e1 = M[nc + id], e2 = M[2 * nc + id];
        dMag[id] = c_scale(mask, c_muli(c_sub(c_scale(ky, e2), c_scale(kz, e1))));
        dMag[nc + id] = c_scale(mask, c_muli(c_sub(c_scale(kz, e0), c_scale(kx, e2))));
        dMag[2 * nc + id] = c_scale(mask, c_muli(c_sub(c_scale(kx, e1), c_scale(ky, e0))));
    }
}

/* ---- Physics::AdvectTemperature (src/physics/boussinesq.cu:10-43) ------ */
static void advect_temperature(orc_ctx* c, const double* rb, cpx* dTh) {
    const size_t nr = c->g.nr, nc = c->g.nc;
    const double* u = rb + (size_t)c->VEL * nr;
    const double* th = rb + (size_t)c->TH * nr;
    double* E = c->rtmp;
    /* EnergyFluxVector (src/cuda/cuda_kernels.cu:277-289) */
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nr; i++) {
        E[i] = u[i] * th[i];
        E[nr + i] = u[nr + i] * th[i];
        E[2 * nr + i] = u[2 * nr + i] * th[i];
    }
    for (int n = 0; n < 3; n++) r2c_3d(&c->g, E + (size_t)n * nr, c->tmp + (size_t)n * nc);
    const cpx* Q = c->tmp;
    /* NonLinBoussinesqAdv (src/cuda/cuda_kernels.cu:293-304): overwrites */
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx a = c_add(c_add(c_scale(kx, Q[id]), c_scale(ky, Q[nc + id])), c_scale(kz, Q[2 * nc + id]));
        dTh[id] = c_scale(-mask, c_muli(a));
    }
}

/* ---- Physics::EntropyStratification (src/physics/boussinesq.cu:46-69),
 *      kernel BoussinesqStrat (src/cuda/cuda_kernels.cu:310-325) --------- */
static void entropy_stratification(orc_ctx* c, const cpx* U, cpx* dU) {
    const size_t nc = c->g.nc;
    const int sd = c->p.strat_direction;
    const cpx* th = U + (size_t)c->TH * nc;
    const cpx* us = U + (size_t)(c->VEL + sd) * nc;
    cpx* dus = dU + (size_t)(c->VEL + sd) * nc;
    cpx* dth = dU + (size_t)c->TH * nc;
    const double N2 = c->p.N2;
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nc; i++) {
        dus[i] = c_sub(dus[i], th[i]);
        dth[i] = c_add(dth[i], c_scale(N2, us[i]));
    }
}

/* ---- nablaOpScalar (src/cuda/cuda_kernels_generic.cu:198-214) ---------- */
static void nabla_op_scalar(orc_ctx* c, const cpx* X, cpx* Z, double a, int accumulate) {
    FOR_MODES(c) {
        MODE_VARS(c)
        double k2 = kx * kx + ky * ky + kz * kz;
        cpx v = c_scale(-a * k2, X[id]);
        Z[id] = accumulate ? c_add(Z[id], v) : v;
    }
}

/* ---- Physics::AnisotropicHeatFlux (src/physics/anisotropic_conduction.cu:10-62)
 * Gradient (cuda_kernels_generic.cu:249-260), 3 C2R, ComputeBGradTheta and
 * ComputeAnisotropicHeatFlux (cuda_kernels.cu:360-383), 3 D2Z,
 * DivergenceMask accumulate (cuda_kernels_generic.cu:315-334). */
static void anisotropic_heat_flux(orc_ctx* c, const cpx* U, const double* rb, cpx* dTh) {
    const size_t nc = c->g.nc, nr = c->g.nr;
    const cpx* th = U + (size_t)c->TH * nc;
    cpx* G = c->tmp;
    FOR_MODES(c) {
        MODE_VARS(c)
        G[id] = c_muli(c_scale(kx, th[id]));
        G[nc + id] = c_muli(c_scale(ky, th[id]));
        G[2 * nc + id] = c_muli(c_scale(kz, th[id]));
    }
    double* g = c->rtmp;  /* gx, gy, gz, then q at [3..5] */
    for (int n = 0; n < 3; n++) c2r_3d(&c->g, G + (size_t)n * nc, g + (size_t)n * nr, c->work);
    const double* B = rb + (size_t)c->MAG * nr;
    const int sd = c->p.strat_direction;
    const double chi = 1. / c->p.reynolds_ani, W = c->p.OmegaT2;
    double* q = c->rtmp + 3 * nr;
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nr; i++) {
        double bx = B[i], by = B[nr + i], bz = B[2 * nr + i];
        double bgt = bx * g[i] + by * g[nr + i] + bz * g[2 * nr + i];
        double b2 = bx * bx + by * by + bz * bz;
        double bs = B[(size_t)sd * nr + i];
        q[i] = chi * bx * (bgt + W * bs) / b2;
        q[nr + i] = chi * by * (bgt + W * bs) / b2;
        q[2 * nr + i] = chi * bz * (bgt + W * bs) / b2;
    }
    for (int n = 0; n < 3; n++) r2c_3d(&c->g, q + (size_t)n * nr, c->tmp + (size_t)n * nc);
    const cpx* Q = c->tmp;
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx a = c_add(c_add(c_scale(kx, Q[id]), c_scale(ky, Q[nc + id])), c_scale(kz, Q[2 * nc + id]));
        dTh[id] = c_add(dTh[id], c_scale(mask, c_muli(a)));
    }
}

/* ---- GradPseudoPressure (src/cuda/cuda_kernels.cu:128-159) ------------- */
static void grad_pseudo_pressure(orc_ctx* c, cpx* dV) {
    const size_t nc = c->g.nc;
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx d0 = dV[id], d1 = dV[nc + id], d2 = dV[2 * nc + id];
        cpx div = c_muli(c_add(c_add(c_scale(kx, d0), c_scale(ky, d1)), c_scale(kz, d2)));
        double k2 = kx * kx + ky * ky + kz * kz;
        double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
        dV[id] = c_add(d0, c_scale(kx * ik2, c_muli(div)));
        dV[nc + id] = c_add(d1, c_scale(ky * ik2, c_muli(div)));
        dV[2 * nc + id] = c_add(d2, c_scale(kz * ik2, c_muli(div)));
    }
}

/* ---- GradPseudoPressureShearing (src/cuda/cuda_kernels.cu:165-196): the
 * divergence of dV carries the background shear's S ky vx ------------- */
static void grad_pseudo_pressure_shearing(orc_ctx* c, cpx* dV, const cpx* Vx) {
    const size_t nc = c->g.nc;
    const double S = c->p.shear;
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx d0 = dV[id], d1 = dV[nc + id], d2 = dV[2 * nc + id];
        cpx div = c_muli(c_add(c_add(c_add(c_scale(S * ky, Vx[id]), c_scale(kx, d0)), c_scale(ky, d1)), c_scale(kz, d2)));
        double k2 = kx * kx + ky * ky + kz * kz;
        double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
        dV[id] = c_add(d0, c_scale(kx * ik2, c_muli(div)));
        dV[nc + id] = c_add(d1, c_scale(ky * ik2, c_muli(div)));
        dV[2 * nc + id] = c_add(d2, c_scale(kz * ik2, c_muli(div)));
    }
}

/* ---- Physics::BackgroundShear / BackgroundRotation
 * (src/physics/shear_rotation.cu:11-63; ShearingFlow and CoriolisForce,
 * cuda_kernels.cu:332-355): dvy += S vx, dBy -= S Bx; with rotation (gated
 * on shearing as in the reference) dvx += 2 omega vy, dvy -= 2 omega vx. */
static void shear_rotation(orc_ctx* c, const cpx* U, cpx* dU) {
    const size_t nc = c->g.nc;
    const double S = c->p.shear, Om = c->p.omega;
    const cpx *vx = U + (size_t)c->VX * nc, *vy = U + (size_t)c->VY * nc;
    cpx *dvx = dU + (size_t)c->VX * nc, *dvy = dU + (size_t)c->VY * nc;
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nc; i++) dvy[i] = c_add(dvy[i], c_scale(S, vx[i]));
    if (c->p.mhd) {
        const cpx* bx = U + (size_t)c->BX * nc;
        cpx* dby = dU + (size_t)c->BY * nc;
        #pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)nc; i++) dby[i] = c_add(dby[i], c_scale(-S, bx[i]));
    }
    if (c->p.rotating) {
        #pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)nc; i++) {
            dvx[i] = c_add(dvx[i], c_scale(2.0 * Om, vy[i]));
            dvy[i] = c_sub(dvy[i], c_scale(2.0 * Om, vx[i]));
        }
    }
}

/* ---- TimeStepping::ShiftTime (src/timestepping/shearing_remapping.cu:15-25) */
static double shift_time(const spk_params_t* p, double t) {
    const double h = p->ly / (2.0 * p->shear * p->lx);
    return fmod(t + h, p->ly / (p->shear * p->lx)) - h;
}

/* ---- TimeStepping::RemapField (shearing_remapping.cu:27-46):
 * RemapComplexVec (cuda_kernels_generic.cu:386-412) moves mode (nx, ny) to
 * nx + ny when that lies strictly inside (-NX/2, NX/2), zero elsewhere;
 * MaskVector (:414-423) then applies the 2/3 mask. */
static void remap_fields(orc_ctx* c) {
    const int NX = c->g.nx, NY = c->g.ny, nzh = c->g.nzh;
    cpx* R = c->tmp;
    for (int f = 0; f < c->F; f++) {
        cpx* X = c->U + (size_t)f * c->g.nc;
        memset(R, 0, sizeof(cpx) * c->g.nc);
        for (int i = 0; i < NX; i++)
            for (int j = 0; j < NY; j++) {
                const int nx = (int)fmod((double)i + (NX / 2), (double)NX) - NX / 2;
                const int ny = (int)fmod((double)j + (NY / 2), (double)NY) - NY / 2;
                int nt = nx + ny;
                if (nt > -NX / 2 && nt < NX / 2) {
                    if (nt < 0) nt += NX;
                    for (int k = 0; k < nzh; k++)
                        R[(size_t)k + (size_t)nzh * ((size_t)j + (size_t)NY * nt)] =
                            X[(size_t)k + (size_t)nzh * ((size_t)j + (size_t)NY * i)];
                }
            }
        FOR_MODES(c) {
            MODE_VARS(c)
            X[id] = c_scale(mask, R[id]);
        }
    }
}

/* End of a step with the shearing module (hydro_mhd_advance.cu:167-180):
 * the remap clock advances by dt; past half a shear period it restarts
 * from the time and the fields are remapped; the wavevector follows. */
static void shear_end_of_step(orc_ctx* c) {
    const spk_params_t* p = &c->p;
    if (!p->shearing) return;
    c->tremap += c->dt;
    if (c->tremap > p->ly / (2.0 * p->shear * p->lx)) {
        c->tremap = shift_time(p, c->t);
        remap_fields(c);
    }
    c->shx = p->shear * c->tremap;
}

/* ---- CleanDivergence (src/cuda/cuda_kernels_generic.cu:288-313) -------- */
static void clean_vec(orc_ctx* c, cpx* X) {
    const size_t nc = c->g.nc;
    FOR_MODES(c) {
        MODE_VARS(c)
        cpx x0 = X[id], x1 = X[nc + id], x2 = X[2 * nc + id];
        cpx q0 = c_muli(c_add(c_add(c_scale(kx, x0), c_scale(ky, x1)), c_scale(kz, x2)));
        double k2 = kx * kx + ky * ky + kz * kz;
        double ik2 = k2 > 0.0 ? 1.0 / k2 : 1.0;
        X[id] = c_add(x0, c_scale(ik2, c_muli(c_scale(kx, q0))));
        X[nc + id] = c_add(x1, c_scale(ik2, c_muli(c_scale(ky, q0))));
        X[2 * nc + id] = c_add(x2, c_scale(ik2, c_muli(c_scale(kz, q0))));
    }
}

/* Fields::CleanFieldDivergence (src/fields/symmetries.cu:114-130) */
void orc_clean_divergence(orc_ctx* c) {
    if (c->p.incompressible) clean_vec(c, c->U + (size_t)c->VEL * c->g.nc);
    if (c->p.mhd) clean_vec(c, c->U + (size_t)c->MAG * c->g.nc);
}

/* ---- TimeStepping::compute_dfield (src/timestepping/compute_dfield.cu:11-90)
 * with Physics::HyperbolicTerms / SourceTerms / ParabolicTerms
 * (src/physics/physics.cu:30-230).  rb must hold C2R(U). */
static void compute_dfield(orc_ctx* c, const cpx* U, const double* rb, cpx* dU) {
    const size_t nc = c->g.nc;
    const spk_params_t* p = &c->p;
    if (p->incompressible) {
        if (c->closure_on) closure_fields(c, U);
        basdevant_hydro(c, rb, dU + (size_t)c->VEL * nc);
        if (p->mhd) curl_emf(c, rb, dU + (size_t)c->MAG * nc);
        if (p->boussinesq) advect_temperature(c, rb, dU + (size_t)c->TH * nc);
        if (p->stratification) entropy_stratification(c, U, dU);
        if (p->shearing) shear_rotation(c, U, dU);
        for (int i = 0; i < 3; i++)
            if (c->sts_pos[c->VEL + i] < 0)
                nabla_op_scalar(c, U + (size_t)(c->VEL + i) * nc, dU + (size_t)(c->VEL + i) * nc, p->nu, 1);
        if (p->mhd)
            for (int i = 0; i < 3; i++)
                if (c->sts_pos[c->MAG + i] < 0)
                    nabla_op_scalar(c, U + (size_t)(c->MAG + i) * nc, dU + (size_t)(c->MAG + i) * nc, p->nu_m, 1);
        if (p->boussinesq && c->sts_pos[c->TH] < 0) {
            if (p->anisotropic_diffusion) anisotropic_heat_flux(c, U, rb, dU + (size_t)c->TH * nc);
            else nabla_op_scalar(c, U + (size_t)c->TH * nc, dU + (size_t)c->TH * nc, p->nu_th, 1);
        }
        if (p->shearing) grad_pseudo_pressure_shearing(c, dU + (size_t)c->VEL * nc, U + (size_t)c->VX * nc);
        else grad_pseudo_pressure(c, dU + (size_t)c->VEL * nc);
    } else if (p->heat_equation) {
        if (c->sts_pos[c->TH] < 0)
            nabla_op_scalar(c, U + (size_t)c->TH * nc, dU + (size_t)c->TH * nc, p->nu_th, 0);
    }
}

void orc_compute_dfield(orc_ctx* c, const double* Uin, double* dUout) {
    const cpx* U = (const cpx*)Uin;
    if (c->p.incompressible) complex2real(c, U, c->realbuf, c->F);
    cpx* dU = c->dU;
    memset(dU, 0, sizeof(cpx) * c->g.nc * c->F);
    compute_dfield(c, U, c->realbuf, dU);
    memcpy(dUout, dU, sizeof(cpx) * c->g.nc * c->F);
}

static double max_abs(const double* a, size_t n) {
    double m = 0.0;
    #pragma omp parallel for reduction(max : m) schedule(static)
    for (long i = 0; i < (long)n; i++) {
        double v = fabs(a[i]);
        if (v > m || v != v) m = v;
    }
    return m;
}

/* ---- TimeStepping::compute_dt (src/timestepping/compute_dt.cu:15-309),
 * with the shearing box's |tremap| ky_max on the x rates and the rotation
 * and shear rates over safety_source (:110-121, 158, 171, 216-220).  The maxima
 * run over the NX*NY*NZ real points (the reference's Idamax also scans the
 * two pad slots of each padded pencil, compute_dt.cu:90-95). */
static void compute_dt(orc_ctx* c) {
    const spk_params_t* p = &c->p;
    double gamma_v = 0.0, gamma_th = 0.0, gamma_par = 0.0, gamma_b = 0.0, gamma_tmp, gamma_sts = 0.0;
    const double kxmax = c->kxmax, kymax = c->kymax, kzmax = c->kzmax;
    double current_dt = c->dt;
    c->dt_hyp = 0.0; c->dt_par = 0.0; c->dt_sts = 0.0;
    if (p->heat_equation) {
        gamma_tmp = ((kxmax) * (kxmax) + kymax * kymax + kzmax * kzmax) * p->nu_th;
        if (c->sts_pos[c->TH] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        c->dt_par = p->cfl * p->cfl_par / gamma_par;
        c->dt_sts = p->cfl_par / gamma_sts;
        current_dt = c->dt_par;
    }
    if (p->incompressible) {
        complex2real(c, c->U, c->realbuf, c->F);
        const size_t nr = c->g.nr;
        const double* rb = c->realbuf;
        double maxfx = max_abs(rb + (size_t)c->VX * nr, nr);
        double maxfy = max_abs(rb + (size_t)c->VY * nr, nr);
        double maxfz = max_abs(rb + (size_t)c->VZ * nr, nr);
        const double kxs = kxmax + fabs(c->tremap) * kymax;
        gamma_v = (kxs * maxfx + kymax * maxfy + kzmax * maxfz);
        if (p->rotating) gamma_v += fabs(p->omega) / p->safety_source;
        if (p->shearing) gamma_v += fabs(p->shear) / p->safety_source;
        gamma_tmp = kxs * kxs * p->nu;
        if (c->sts_pos[c->VX] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kymax * kymax * p->nu;
        if (c->sts_pos[c->VY] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        gamma_tmp = kzmax * kzmax * p->nu;
        if (c->sts_pos[c->VZ] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        if (p->boussinesq) {
            gamma_th += pow(fabs(p->N2), 0.5) / p->safety_source;
            if (p->anisotropic_diffusion) {
                gamma_th += pow(fabs(p->OmegaT2), 0.5) / p->safety_source;
                gamma_tmp = (kxs * kxs + kymax * kymax + kzmax * kzmax) * (1. / p->reynolds_ani);
            } else {
                gamma_tmp = (kxs * kxs + kymax * kymax + kzmax * kzmax) * p->nu_th;
            }
            if (c->sts_pos[c->TH] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        }
        if (p->mhd) {
            double maxbx = max_abs(rb + (size_t)c->BX * nr, nr);
            double maxby = max_abs(rb + (size_t)c->BY * nr, nr);
            double maxbz = max_abs(rb + (size_t)c->BZ * nr, nr);
            gamma_b = kxs * maxbx + kymax * maxby + kzmax * maxbz;
            gamma_tmp = kxs * kxs * p->nu_m;
            if (c->sts_pos[c->BX] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kymax * kymax * p->nu_m;
            if (c->sts_pos[c->BY] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
            gamma_tmp = kzmax * kzmax * p->nu_m;
            if (c->sts_pos[c->BZ] < 0) gamma_par += gamma_tmp; else gamma_sts += gamma_tmp;
        }
        if (c->closure_on) {
            /* the closure's eddy viscosity and resistivity as parabolic rates */
            closure_fields(c, c->U);
            const double k2 = kxmax * kxmax + kymax * kymax + kzmax * kzmax;
            gamma_par += k2 * c->nu_t_max;
            if (p->mhd) gamma_par += k2 * c->eta_t_max;
        }
        c->dt_hyp = p->cfl / (gamma_v + gamma_th + gamma_b);
        c->dt_par = p->cfl_par / gamma_par;
        c->dt_sts = p->cfl_sts / gamma_sts;
        current_dt = (c->dt_hyp < c->dt_par) ? c->dt_hyp : c->dt_par;
        if (p->supertimestepping) {
            if (current_dt > c->dt_sts * p->safety_sts) current_dt = c->dt_sts * p->safety_sts;
        }
    }
    if (p->fixed_dt > 0.0) current_dt = p->fixed_dt;
    if (c->t + current_dt > p->t_final) current_dt = p->t_final - c->t;
    else if (c->t + current_dt - c->t_lastsnap > p->toutput_flow) current_dt = p->toutput_flow - c->t + c->t_lastsnap;
    if (p->supertimestepping) {
        if (c->dt_sts > current_dt) c->dt_sts = current_dt;
    }
    c->dt = current_dt;
}

void orc_compute_dt(orc_ctx* c, double out4[4]) {
    compute_dt(c);
    out4[0] = c->dt_hyp; out4[1] = c->dt_par; out4[2] = c->dt_sts; out4[3] = c->dt;
}

/* ---- Physics::ParabolicTermsSTS (src/physics/physics.cu:233-330): sets
 * the RHS of the STS variables into dsts[pos] (zeroed by the caller).
 * B-field STS with anisotropic conduction re-transforms B into rb first. */
static void parabolic_terms_sts(orc_ctx* c, const cpx* U, double* rb, cpx* dsts) {
    const size_t nc = c->g.nc;
    const spk_params_t* p = &c->p;
    if (p->incompressible)
        for (int i = 0; i < 3; i++)
            if (c->sts_pos[c->VEL + i] >= 0)
                nabla_op_scalar(c, U + (size_t)(c->VEL + i) * nc, dsts + (size_t)c->sts_pos[c->VEL + i] * nc, p->nu, 0);
    if (p->mhd)
        for (int i = 0; i < 3; i++)
            if (c->sts_pos[c->MAG + i] >= 0)
                nabla_op_scalar(c, U + (size_t)(c->MAG + i) * nc, dsts + (size_t)c->sts_pos[c->MAG + i] * nc, p->nu_m, 0);
    if ((p->boussinesq || p->heat_equation) && c->sts_pos[c->TH] >= 0) {
        cpx* dth = dsts + (size_t)c->sts_pos[c->TH] * nc;
        if (p->anisotropic_diffusion) {
            for (int i = 0; i < 3; i++)
                if (c->sts_pos[c->MAG + i] >= 0)
                    c2r_3d(&c->g, U + (size_t)(c->MAG + i) * nc, rb + (size_t)(c->MAG + i) * c->g.nr, c->work);
            anisotropic_heat_flux(c, U, rb, dth);
        } else {
            nabla_op_scalar(c, U + (size_t)c->TH * nc, dth, p->nu_th, 0);
        }
    }
}

/* ---- STS_FindRoot / STS_CorrectTimeStep / STS_ComputeSubSteps
 * (src/rkl/rkl.cu:594-664): the sub-step sequence of Alexiades, Amiez &
 * Gremaud (1996), damping STS_NU = 0.001 (src/rkl/rkl.hpp:32). */
#define ORC_STS_NU 0.001
#define ORC_STS_MAX_STEPS 1024   /* src/rkl/rkl.hpp:30 */
static double sts_find_root(double dt_exp, double dT, double nu) {
    const double sq = sqrt(nu), a = (1.0 - sq) / (1.0 + sq);
    double N = 1.0;
    for (int k = 0; k < 128; k++) {
        const double b = pow(a, 2.0 * N);
        const double cc = (1.0 - b) / (1.0 + b);
        const double db_dN = 2.0 * log(a) * b;
        const double scrh = cc - N * 2.0 / ((1.0 + b) * (1.0 + b)) * db_dN;
        const double fN = dT - 0.5 * dt_exp / sq * N * cc;
        const double dfN = -0.5 * dt_exp / sq * scrh;
        const double dN = fN / dfN;
        N -= dN;
        if (fabs(dN) < 1.e-5) return N;
    }
    return -1.0;
}
static double sts_correct_dt(int n0, double dta, double nu) {
    const double a = (1.0 - sqrt(nu)) / (1.0 + sqrt(nu));
    const double b = pow(a, 2.0 * n0), cc = (1.0 - b) / (1.0 + b);
    return dta * 2.0 * sqrt(nu) / (n0 * cc);
}

/* ---- RKLegendre::compute_cycle_STS (src/rkl/rkl.cu:207-283): n sub-steps
 * U <- U + tau dU (addReset, src/cuda/cuda_kernels_generic.cu:174-181), taken
 * in the reverse order of the sequence.  Returns n, or -1 when the root
 * search fails or n exceeds STS_MAX_STEPS (the reference reads outside its
 * sub-step array there). */
static int sts_cycle(orc_ctx* c) {
    const size_t nc = c->g.nc;
    const int ns = c->nsts;
    const double dt_current = c->dt, dt_sts = c->dt_sts;
    const int n = (int)floor(sts_find_root(dt_sts, dt_current, ORC_STS_NU) + 1.0);
    if (n < 1 || n > ORC_STS_MAX_STEPS) return -1;
    double* ts = (double*)calloc((size_t)n, sizeof(double));
    if (n > 1) {
        const double dtc = sts_correct_dt(n, dt_current, ORC_STS_NU);
        for (int i = 0; i < n; i++)
            ts[i] = dtc / ((-1.0 + ORC_STS_NU) * cos(((2.0 * i + 1.0) * M_PI) / (2.0 * n)) + 1.0 + ORC_STS_NU);
    } else {
        ts[0] = dt_current;
    }
    for (int m = 0; m < n; m++) {
        const double tau = ts[n - m - 1];
        memset(c->rdU, 0, sizeof(cpx) * nc * ns);
        parabolic_terms_sts(c, c->U, c->realbuf, c->rdU);
        for (int nv = 0; nv < ns; nv++) {
            cpx* Uc = c->U + (size_t)c->sts_index[nv] * nc;
            cpx* dU = c->rdU + (size_t)nv * nc;
            #pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)nc; i++) {
                Uc[i] = c_add(c_scale(1.0, Uc[i]), c_scale(tau, dU[i]));
                dU[i] = (cpx){0.0, 0.0};
            }
        }
    }
    free(ts);
    return n;
}

/* ---- RKLegendre::compute_cycle_RKL1 (src/rkl/rkl.cu:286-434) ----------- */
static int rkl1_cycle(orc_ctx* c) {
    const size_t nc = c->g.nc;
    const int ns = c->nsts;
    const double dt_current = c->dt, dt_sts = c->dt_sts;
    const double scrh = dt_current / dt_sts;
    const double s_str = 4.0 * scrh / (1.0 + sqrt(1.0 + 8.0 * scrh));
    const int s_RKL = 1 + (int)(s_str);
    const double w1 = 2.0 / (s_RKL * s_RKL + s_RKL);
    double mu_tilde_j = w1;
    memset(c->rdU0, 0, sizeof(cpx) * nc * ns);
    memset(c->rdU, 0, sizeof(cpx) * nc * ns);
    parabolic_terms_sts(c, c->U, c->realbuf, c->rdU);
    for (int nv = 0; nv < ns; nv++) {
        cpx* Uc = c->U + (size_t)c->sts_index[nv] * nc;
        cpx *Uc0 = c->rUc0 + (size_t)nv * nc, *Uc1 = c->rUc1 + (size_t)nv * nc;
        cpx *dU = c->rdU + (size_t)nv * nc, *dU0 = c->rdU0 + (size_t)nv * nc;
        #pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)nc; i++) {
            Uc0[i] = Uc[i];
            dU0[i] = dU[i];
            Uc1[i] = Uc[i];
            Uc[i] = c_add(c_scale(1.0, Uc1[i]), c_scale(mu_tilde_j * dt_current, dU0[i]));
        }
    }
    for (int stage = 2; stage <= s_RKL; stage++) {
        const double mu_j = (2. * stage - 1.) / stage;
        mu_tilde_j = w1 * mu_j;
        const double nu_j = -(stage - 1.) / stage;
        memset(c->rdU, 0, sizeof(cpx) * nc * ns);
        parabolic_terms_sts(c, c->U, c->realbuf, c->rdU);
        for (int nv = 0; nv < ns; nv++) {
            cpx* Uc = c->U + (size_t)c->sts_index[nv] * nc;
            cpx* Uc1 = c->rUc1 + (size_t)nv * nc;
            cpx* dU = c->rdU + (size_t)nv * nc;
            const double a = dt_current * mu_tilde_j;
            /* rkl1_stage (src/cuda/cuda_kernels_generic.cu:146-158) */
            #pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)nc; i++) {
                cpx Y = c_add(c_scale(mu_j, Uc[i]), c_scale(nu_j, Uc1[i]));
                Uc1[i] = Uc[i];
                Uc[i] = c_add(Y, c_scale(a, dU[i]));
            }
        }
    }
    return s_RKL;
}

/* ---- RKLegendre::compute_cycle_RKL2 (src/rkl/rkl.cu:437-591) ----------- */
static int rkl2_cycle(orc_ctx* c) {
    const size_t nc = c->g.nc;
    const int ns = c->nsts;
    const double dt_current = c->dt, dt_sts = c->dt_sts;
    double scrh = dt_current / dt_sts;
    double s_str = 4.0 * (1.0 + 2.0 * scrh) / (1.0 + sqrt(9.0 + 16.0 * scrh));
    int s_RKL = 1 + (int)(s_str);
    double w1 = 4.0 / (s_RKL * s_RKL + s_RKL - 2.0);
    double mu_tilde_j = w1 / 3.0;
    double b_j, b_jm1, b_jm2, a_jm1;
    b_j = b_jm1 = b_jm2 = 1.0 / 3.0;
    a_jm1 = 1.0 - b_jm1;
    memset(c->rdU0, 0, sizeof(cpx) * nc * ns);
    memset(c->rdU, 0, sizeof(cpx) * nc * ns);
    parabolic_terms_sts(c, c->U, c->realbuf, c->rdU);
    for (int nv = 0; nv < ns; nv++) {
        cpx* Uc = c->U + (size_t)c->sts_index[nv] * nc;
        cpx *Uc0 = c->rUc0 + (size_t)nv * nc, *Uc1 = c->rUc1 + (size_t)nv * nc;
        cpx *dU = c->rdU + (size_t)nv * nc, *dU0 = c->rdU0 + (size_t)nv * nc;
        #pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)nc; i++) {
            Uc0[i] = Uc[i];
            dU0[i] = dU[i];
            Uc1[i] = Uc[i];
            Uc[i] = c_add(c_scale(1.0, Uc1[i]), c_scale(mu_tilde_j * dt_current, dU0[i]));
        }
    }
    for (int stage = 2; stage <= s_RKL; stage++) {
        double mu_j = (2. * stage - 1.) / stage * b_j / b_jm1;
        mu_tilde_j = w1 * mu_j;
        double gamma_j = -a_jm1 * mu_tilde_j;
        double nu_j = -(stage - 1.) * b_j / (stage * b_jm2);
        memset(c->rdU, 0, sizeof(cpx) * nc * ns);
        parabolic_terms_sts(c, c->U, c->realbuf, c->rdU);
        for (int nv = 0; nv < ns; nv++) {
            cpx* Uc = c->U + (size_t)c->sts_index[nv] * nc;
            cpx *Uc0 = c->rUc0 + (size_t)nv * nc, *Uc1 = c->rUc1 + (size_t)nv * nc;
            cpx *dU = c->rdU + (size_t)nv * nc, *dU0 = c->rdU0 + (size_t)nv * nc;
            const double a = dt_current * mu_tilde_j, gdt = gamma_j * dt_current, cm = (1.0 - mu_j - nu_j);
            /* rkl2_stage (src/cuda/cuda_kernels_generic.cu:160-172) */
            #pragma omp parallel for schedule(static)
            for (long i = 0; i < (long)nc; i++) {
                cpx Y = c_add(c_scale(mu_j, Uc[i]), c_scale(nu_j, Uc1[i]));
                Uc1[i] = Uc[i];
                Uc[i] = c_add(c_add(c_add(Y, c_scale(cm, Uc0[i])), c_scale(a, dU[i])), c_scale(gdt, dU0[i]));
            }
        }
        b_jm2 = b_jm1;
        b_jm1 = b_j;
        a_jm1 = 1.0 - b_jm1;
        b_j = 0.5 * (stage * stage + 3.0 * stage) / (stage * stage + 3.0 * stage + 2);
    }
    return s_RKL;
}

/* RKLegendre::compute_cycle (src/rkl/rkl.cu:185-199) */
static int sts_dispatch(orc_ctx* c) {
    if (c->p.sts_algorithm == SPK_STS_STS) return sts_cycle(c);
    if (c->p.sts_algorithm == SPK_STS_RKL1) return rkl1_cycle(c);
    return rkl2_cycle(c);
}

int orc_rkl_cycle(orc_ctx* c) {
    if (c->nsts == 0) return 0;
    return sts_dispatch(c);
}

/* axpyComplex (src/cuda/cuda_kernels_generic.cu:137-144): Z = a X + b Y */
static void axpy(const cpx* X, const cpx* Y, cpx* Z, double a, double b, size_t n) {
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) Z[i] = c_add(c_scale(a, X[i]), c_scale(b, Y[i]));
}

/* ---- TimeStepping::RungeKutta3 (src/timestepping/hydro_mhd_advance.cu:79-189) */
static void runge_kutta3(orc_ctx* c) {
    static const double gammaRK[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    static const double xiRK[2] = {-17.0 / 60.0, -5.0 / 12.0};
    const size_t n = c->g.nc * c->F;
    const double dt = c->dt;
    cpx *U = c->U, *dU = c->dU, *S = c->S;
    /* stage 1: real buffer from compute_dt */
    const int sh = c->p.shearing;
    compute_dfield(c, U, c->realbuf, dU);
    axpy(U, dU, U, 1.0, gammaRK[0] * dt, n);
    axpy(U, dU, S, 1.0, xiRK[0] * dt, n);
    if (c->p.incompressible) complex2real(c, U, c->realbuf, c->F);
    if (sh) c->shx = c->p.shear * (c->tremap + gammaRK[0] * dt);
    compute_dfield(c, U, c->realbuf, dU);
    axpy(S, dU, U, 1.0, gammaRK[1] * dt, n);
    axpy(U, dU, S, 1.0, xiRK[1] * dt, n);
    if (c->p.incompressible) complex2real(c, U, c->realbuf, c->F);
    if (sh) c->shx = c->p.shear * (c->tremap + (gammaRK[0] + xiRK[0] + gammaRK[1]) * dt);
    compute_dfield(c, U, c->realbuf, dU);
    axpy(S, dU, U, 1.0, gammaRK[2] * dt, n);
    c->t += c->dt;
    shear_end_of_step(c);
}

/* ---- TimeStepping::ForwardEuler (hydro_mhd_advance.cu:191-248) -------- */
static void forward_euler(orc_ctx* c) {
    const size_t n = c->g.nc * c->F;
    compute_dfield(c, c->U, c->realbuf, c->dU);
    axpy(c->U, c->dU, c->U, 1.0, c->dt, n);
    c->t += c->dt;
    shear_end_of_step(c);
}

/* ---- one main-loop iteration: Supervisor::executeMainLoop body
 * (src/supervisor/supervisor.cu:179-192) = CleanFieldDivergence +
 * TimeStepping::HydroMHDAdvance (hydro_mhd_advance.cu:18-75). */
void orc_step(orc_ctx* c, int nsteps) {
    const spk_params_t* p = &c->p;
    for (int it = 0; it < nsteps; it++) {
        orc_clean_divergence(c);
        compute_dt(c);
        if (p->sts_every_step) {
            if (p->integrator == SPK_INT_EULER) forward_euler(c); else runge_kutta3(c);
            if (p->supertimestepping) {
                if (p->incompressible) complex2real(c, c->U, c->realbuf, c->F);
                sts_dispatch(c);
            }
        } else {
            if (p->supertimestepping && (c->step % 2) == 1) sts_dispatch(c);
            if (p->integrator == SPK_INT_EULER) forward_euler(c); else runge_kutta3(c);
            if (p->supertimestepping && (c->step % 2) == 0) {
                if (p->incompressible) complex2real(c, c->U, c->realbuf, c->F);
                sts_dispatch(c);
            }
        }
        c->step += 1;
    }
}

/* Spectral products of U before their divergence / curl (hydro.cu:19-75,
 * mhd.cu:20-62 up to the R2C), closure terms included when on; modes
 * outside the 2/3 mask set to zero.  P: [nprod][Nc], nprod 5 (HD) or 8 (MHD). */
int orc_products(orc_ctx* c, const double* Uin, double* Pout) {
    const cpx* U = (const cpx*)Uin;
    cpx* P = (cpx*)Pout;
    const size_t nr = c->g.nr, nc = c->g.nc;
    if (!c->p.incompressible) return 0;
    complex2real(c, U, c->realbuf, c->F);
    if (c->closure_on) closure_fields(c, U);
    const int mhd = c->p.mhd, np = mhd ? 8 : 5;
    double* R = (double*)calloc(nr * np, sizeof(double));
    const double* u = c->realbuf + (size_t)c->VEL * nr;
    const double* B = c->realbuf + (size_t)c->MAG * nr;
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nr; i++) {
        const double ux = u[i], uy = u[nr + i], uz = u[2 * nr + i];
        const double bx = mhd ? B[i] : 0.0, by = mhd ? B[nr + i] : 0.0, bz = mhd ? B[2 * nr + i] : 0.0;
        R[i] = (2.0 * ux * ux - uy * uy - uz * uz - 2.0 * bx * bx + by * by + bz * bz) / 3.0;
        R[nr + i] = ux * uy - bx * by;
        R[2 * nr + i] = ux * uz - bx * bz;
        R[3 * nr + i] = (-ux * ux + 2.0 * uy * uy - uz * uz + bx * bx - 2.0 * by * by + bz * bz) / 3.0;
        R[4 * nr + i] = uy * uz - by * bz;
        if (mhd) {
            R[5 * nr + i] = -by * uz + bz * uy;
            R[6 * nr + i] = bx * uz - bz * ux;
            R[7 * nr + i] = -bx * uy + by * ux;
        }
    }
    if (c->closure_on)
        for (size_t i = 0; i < (size_t)np * nr; i++) R[i] += c->rclos[i];
    for (int n = 0; n < np; n++) {
        r2c_3d(&c->g, R + (size_t)n * nr, P + (size_t)n * nc);
        cpx* X = P + (size_t)n * nc;
        FOR_MODES(c) {
            MODE_VARS(c)
            if (mask == 0.0) { X[id].re = 0.0; X[id].im = 0.0; }
        }
    }
    free(R);
    return np;
}

/* Sharp spectral filter: the coarse grid's kept modes of fine-grid spectra
 * (scaled by the point-count ratio, since the forward transform is
 * unnormalised), zero elsewhere. */
void orc_truncate(const orc_ctx* f, const orc_ctx* c, const double* Xf, int nch, double* Xc) {
    const double scale = (double)c->g.nr / (double)f->g.nr;
    for (int ch = 0; ch < nch; ch++) {
        const cpx* A = (const cpx*)Xf + (size_t)ch * f->g.nc;
        cpx* Bc = (cpx*)Xc + (size_t)ch * c->g.nc;
        FOR_MODES(c) {
            MODE_VARS(c)
            cpx v = {0.0, 0.0};
            if (mask != 0.0) {
                const int ix = i_ < c->g.nx / 2 ? i_ : i_ - c->g.nx, iy = j_ < c->g.ny / 2 ? j_ : j_ - c->g.ny;
                const int fi = ix >= 0 ? ix : ix + f->g.nx, fj = iy >= 0 ? iy : iy + f->g.ny;
                v = c_scale(scale, A[(size_t)k_ + f->g.nzh * ((size_t)fj + (size_t)fi * f->g.ny)]);
            }
            Bc[id] = v;
        }
    }
}

/* Training samples (include/spooky_b200.h, spk_closure_samples): one per
 * coarse point, rows of SPK_CLOSURE_ROWS doubles (variant 3: SPK_CLOSURE3_ROWS) `stride` apart.  The coarse
 * context's state becomes the filtered fine state. */
void orc_closure_samples(orc_ctx* f, const double* Uf, orc_ctx* c, double* X, size_t stride) {
    const size_t nr = c->g.nr, nc = c->g.nc;
    const int np = c->p.mhd ? 8 : 5;
    const int fon = f->closure_on, con = c->closure_on;
    f->closure_on = 0;
    c->closure_on = 0;
    double* Pf = (double*)malloc(sizeof(cpx) * f->g.nc * np);
    double* Pt = (double*)malloc(sizeof(cpx) * nc * np);
    double* Pc = (double*)malloc(sizeof(cpx) * nc * np);
    orc_products(f, Uf, Pf);
    orc_truncate(f, c, Uf, c->F, (double*)c->U);
    orc_truncate(f, c, Pf, np, Pt);
    orc_products(c, (const double*)c->U, Pc);
    for (size_t i = 0; i < 2 * nc * np; i++) Pt[i] -= Pc[i];
    double* Rt = (double*)malloc(sizeof(double) * nr * np);
    for (int n = 0; n < np; n++) c2r_3d(&c->g, (const cpx*)Pt + (size_t)n * nc, Rt + (size_t)n * nr, c->work);
    if (!c->rgrad) {
        c->rclos = (double*)calloc(nr * 8, sizeof(double));
        c->rgrad = (double*)calloc(nr * 18, sizeof(double));
        c->ctmp = (cpx*)calloc(nc, sizeof(cpx));
    }
    /* strain and current of the whole resolved field, then the model's gradients */
    double* full = (double*)malloc(sizeof(double) * nr * 8);
    closure_grads(c, c->U, 0);
    #pragma omp parallel for schedule(static)
    for (long q = 0; q < (long)nr; q++) {
        double A[9], G[9], fe[8], S5[5], J3[3];
        for (int r = 0; r < 9; r++) { A[r] = c->rgrad[(size_t)r * nr + q]; G[r] = c->rgrad[(size_t)(9 + r) * nr + q]; }
        orc_closure_features(A, G, fe, S5, J3);
        for (int r = 0; r < 5; r++) full[(size_t)r * nr + q] = S5[r];
        for (int r = 0; r < 3; r++) full[(size_t)(5 + r) * nr + q] = J3[r];
    }
    closure_grads(c, c->U, c->p.closure == 2);
    #pragma omp parallel for schedule(static)
    for (long q = 0; q < (long)nr; q++) {
        double A[9], G[9], fe[8], S5[5], J3[3];
        for (int r = 0; r < 9; r++) { A[r] = c->rgrad[(size_t)r * nr + q]; G[r] = c->rgrad[(size_t)(9 + r) * nr + q]; }
        const double n = orc_closure_features(A, G, fe, S5, J3);
        for (int r = 0; r < 8; r++) X[(size_t)(SPK_CLOSURE_ROW_FEAT + r) * stride + q] = fe[r];
        for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_S + r) * stride + q] = S5[r];
        for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_J + r) * stride + q] = J3[r];
        X[(size_t)SPK_CLOSURE_ROW_SCALE * stride + q] = c->delta2 * n;
        for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_TT + r) * stride + q] = Rt[(size_t)r * nr + q];
        for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_TE + r) * stride + q] = np == 8 ? Rt[(size_t)(5 + r) * nr + q] : 0.0;
        for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_SF + r) * stride + q] = full[(size_t)r * nr + q];
        for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_JF + r) * stride + q] = full[(size_t)(5 + r) * nr + q];
        if (c->p.closure == 3)
            for (int r = 0; r < 9; r++) {
                X[(size_t)(SPK_CLOSURE_ROW_A + r) * stride + q] = A[r];
                X[(size_t)(SPK_CLOSURE_ROW_G + r) * stride + q] = G[r];
            }
    }
    free(full);
    free(Pf); free(Pt); free(Pc); free(Rt);
    f->closure_on = fon;
    c->closure_on = con;
}

void orc_to_real(orc_ctx* c, double* R) { complex2real(c, c->U, R, c->F); }

void orc_r2c(orc_ctx* c, const double* R, double* C) { r2c_3d(&c->g, R, (cpx*)C); }
void orc_c2r(orc_ctx* c, const double* C, double* R) { c2r_3d(&c->g, (const cpx*)C, R, c->work); }

/* computeEnergy (src/io/spooky_output_functions.cu:23-55): half-spectrum
 * double counting, 0.5 * (2 sum|q|^2 - sum_{kz=0}|q|^2) / N^6; the
 * dissipation weights each mode by k^2. */
void orc_budgets(orc_ctx* c, double* energy, double* dissipation) {
    const size_t nc = c->g.nc;
    const double n2 = (double)c->g.nr * (double)c->g.nr;
    for (int f = 0; f < c->F; f++) {
        const cpx* q = c->U + (size_t)f * nc;
        double e = 0.0, d = 0.0;
        #pragma omp parallel for collapse(2) reduction(+ : e, d) schedule(static)
        for (int i = 0; i < c->g.nx; i++)
            for (int j = 0; j < c->g.ny; j++)
                for (int k = 0; k < c->g.nzh; k++) {
                    size_t id = (size_t)k + c->g.nzh * ((size_t)j + (size_t)i * c->g.ny);
                    double w = (k == 0) ? 1.0 : 2.0;
                    double a2 = q[id].re * q[id].re + q[id].im * q[id].im;
                    double k2 = c->kx[i] * c->kx[i] + c->ky[j] * c->ky[j] + c->kz[k] * c->kz[k];
                    e += w * a2;
                    d += w * k2 * a2;
                }
        energy[f] = 0.5 * e / n2;
        dissipation[f] = d / n2;
    }
}
