/*
 * spk_closure.h -- CPU FP64 restatement of the learned subgrid closure.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA closure kernels
 * (features, MLP inference, loss gradient, Adam).  The closure has no
 * counterpart in the reference; its definition is the one stated in
 * include/spooky_b200.h (SPK_CLOSURE_*).
 */
#ifndef SPK_CLOSURE_ORACLE_H
#define SPK_CLOSURE_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A[3*i+j] = d u_i / d x_j, G likewise for B.  Writes the 8 features, the
 * strain S (xx xy xz yy yz), the current J and returns n. */
double orc_closure_features(const double* A, const double* G, double* feat, double* S5, double* J3);

/* MLP outputs o[2] for features f[8]; nu = scale * softplus(o0), eta = scale * softplus(o1). */
void orc_closure_mlp(const double* params, const double* f, double* o);

/* Mean loss and its gradient over samples rows (SoA, row r at samples + r*stride);
 * w[0], w[1], w[2]: weights of the stress, EMF and energy-transfer errors. */
void orc_closure_loss_grad(const double* samples, size_t n, size_t stride, const double* params,
                           const double* w, double* grad, double* loss);

/* One Adam step (t >= 1) with beta1 0.9, beta2 0.999, eps 1e-8. */
void orc_closure_adam(double* params, const double* grad, double* m, double* v, int t, double lr);

/* Variant 3, the tensor network (SPK_CLOSURE3_*): outputs o[12] for the
 * dimensionless gradients x[18]; the RHS terms of one point (ramp
 * included; returns n); mean loss and gradient over samples with
 * SPK_CLOSURE3_ROWS rows; rounding 0 drops every BF16 rounding. */
void orc_closure3_set_rounding(int on);
void orc_closure3_mlp(const double* params, const double* x, double* o);
double orc_closure3_terms(const double* params, double delta2, const double* A, const double* G, int mhd, double* tau5,
                          double* e3, double* nu_eff, double* eta_eff);
void orc_closure3_loss_grad(const double* samples, size_t n, size_t stride, const double* params, const double* w,
                            double* grad, double* loss);
/* Adam over np parameters (orc_closure_adam: np = SPK_CLOSURE_NPARAM). */
void orc_closure_adam_n(double* params, const double* grad, double* m, double* v, int t, double lr, int np);

#ifdef __cplusplus
}
#endif
#endif
