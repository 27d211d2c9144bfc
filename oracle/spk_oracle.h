/*
 * spk_oracle.h -- CPU FP64 restatement of SPOOKY's RHS + RK3/RKL2 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  The product path never calls it.
 *
 * Each function cites the reference (LorenzoLMP/spooky-git) file:line whose
 * algorithm it restates.  The FFT is the oracle's own mixed-radix Stockham
 * transform written from the DFT definition (the reference calls cuFFT,
 * src/cuda/cufft_routines.cu:17,35,92-93); it is checked against numpy.fft.
 */
#ifndef SPK_ORACLE_H
#define SPK_ORACLE_H
#include <stddef.h>
#include "../include/spooky_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(const spk_params_t* p);
void     orc_destroy(orc_ctx* c);
int      orc_num_fields(const orc_ctx* c);
size_t   orc_ncomplex(const orc_ctx* c);

void orc_set_state(orc_ctx* c, const double* U);     /* [F][Nc] complex */
void orc_get_state(const orc_ctx* c, double* U);
void orc_set_time(orc_ctx* c, double t, int step, double t_lastsnap);
double orc_get_tremap(const orc_ctx* c);
void orc_get_time(const orc_ctx* c, double* t, double* dt, int* step);

/* k tables: kvec[3][Nc] and mask[Nc], plus kxmax, kymax, kzmax, kmax. */
void orc_kgrid(const orc_ctx* c, double* kvec, double* mask, double* kmax4);

void orc_clean_divergence(orc_ctx* c);
void orc_compute_dt(orc_ctx* c, double out4[4]);           /* dt_hyp, dt_par, dt_sts, dt */
void orc_compute_dfield(orc_ctx* c, const double* U, double* dU);
void orc_step(orc_ctx* c, int nsteps);                      /* clean + HydroMHDAdvance */
int  orc_rkl_cycle(orc_ctx* c);                             /* returns the stage count */
void orc_to_real(orc_ctx* c, double* R);                    /* F * NX*NY*NZ */
void orc_budgets(orc_ctx* c, double* energy, double* dissipation);

/* Transforms in the reference's conventions (for FFT tests):
 * r2c: unnormalised forward; c2r: input pre-scaled by 1/(NX NY NZ). */
void orc_r2c(orc_ctx* c, const double* R, double* C);
void orc_c2r(orc_ctx* c, const double* C, double* R);
/* 1-D complex FFT of length n (sign -1 forward, +1 inverse, unnormalised). */
void orc_fft1d(int n, const double* in, double* out, int sign);

void orc_set_threads(int nthreads);

/* Learned closure (include/spooky_b200.h, SPK_CLOSURE_*): params NULL = off;
 * returns nonzero for contexts other than HD / MHD. */
int  orc_closure_set(orc_ctx* c, const double* params);
int  orc_products(orc_ctx* c, const double* U, double* P);   /* returns nprod */
void orc_truncate(const orc_ctx* fine, const orc_ctx* coarse, const double* Xf, int nch, double* Xc);
void orc_closure_samples(orc_ctx* fine, const double* Uf, orc_ctx* coarse, double* X, size_t stride);

#ifdef __cplusplus
}
#endif
#endif
