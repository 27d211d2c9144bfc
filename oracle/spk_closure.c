/*
 * spk_closure.c -- CPU FP64 restatement of the learned subgrid closure.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA closure kernels).  The
 * closure is this project's own (no reference counterpart); this file
 * follows its definition in include/spooky_b200.h, written independently of
 * the CUDA kernels: plain loops in FP64.
 */
#include "spk_closure.h"

#include <math.h>
#include <string.h>

#include "../include/spooky_b200.h"

enum { NF = SPK_CLOSURE_NFEAT, NH = SPK_CLOSURE_HIDDEN, NO = 2 };
/* parameter offsets */
enum { OW1 = 0, OB1 = OW1 + NH * NF, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NO * NH };

double orc_closure_features(const double* A, const double* G, double* f, double* S5, double* J3) {
    double S[3][3], SB[3][3], w[3], J[3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            S[i][j] = 0.5 * (A[3 * i + j] + A[3 * j + i]);
            SB[i][j] = 0.5 * (G[3 * i + j] + G[3 * j + i]);
        }
    /* curl: w_i = eps_ijk d_j u_k */
    w[0] = A[3 * 2 + 1] - A[3 * 1 + 2];
    w[1] = A[3 * 0 + 2] - A[3 * 2 + 0];
    w[2] = A[3 * 1 + 0] - A[3 * 0 + 1];
    J[0] = G[3 * 2 + 1] - G[3 * 1 + 2];
    J[1] = G[3 * 0 + 2] - G[3 * 2 + 0];
    J[2] = G[3 * 1 + 0] - G[3 * 0 + 1];
    double s2 = 0, b2 = 0, w2 = 0, j2 = 0, tr3 = 0, wsw = 0, jsj = 0, wj = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            s2 += S[i][j] * S[i][j];
            b2 += SB[i][j] * SB[i][j];
            wsw += w[i] * S[i][j] * w[j];
            jsj += J[i] * S[i][j] * J[j];
            for (int k = 0; k < 3; k++) tr3 += S[i][j] * S[j][k] * S[k][i];
        }
    for (int i = 0; i < 3; i++) {
        w2 += 0.5 * w[i] * w[i];
        j2 += 0.5 * J[i] * J[i];
        wj += w[i] * J[i];
    }
    const double n2 = s2 + w2 + b2 + j2 + 1e-30;
    const double n = sqrt(n2);
    f[0] = s2 / n2;
    f[1] = w2 / n2;
    f[2] = b2 / n2;
    f[3] = j2 / n2;
    f[4] = tr3 / (n2 * n);
    f[5] = wsw / (n2 * n);
    f[6] = jsj / (n2 * n);
    f[7] = wj * wj / (4.0 * n2 * n2);
    S5[0] = S[0][0]; S5[1] = S[0][1]; S5[2] = S[0][2]; S5[3] = S[1][1]; S5[4] = S[1][2];
    J3[0] = J[0]; J3[1] = J[1]; J3[2] = J[2];
    return n;
}

static void forward(const double* P, const double* f, double* h1, double* h2, double* o) {
    for (int j = 0; j < NH; j++) {
        double a = P[OB1 + j];
        for (int i = 0; i < NF; i++) a += P[OW1 + j * NF + i] * f[i];
        h1[j] = tanh(a);
    }
    for (int j = 0; j < NH; j++) {
        double a = P[OB2 + j];
        for (int i = 0; i < NH; i++) a += P[OW2 + j * NH + i] * h1[i];
        h2[j] = tanh(a);
    }
    for (int j = 0; j < NO; j++) {
        double a = P[OB3 + j];
        for (int i = 0; i < NH; i++) a += P[OW3 + j * NH + i] * h2[i];
        o[j] = a;
    }
}

void orc_closure_mlp(const double* params, const double* f, double* o) {
    double h1[NH], h2[NH];
    forward(params, f, h1, h2, o);
}

static double softplus(double x) { return x > 30.0 ? x : log1p(exp(x)); }
static double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

void orc_closure_loss_grad(const double* X, size_t n, size_t stride, const double* P, const double* w,
                           double* grad, double* loss) {
    memset(grad, 0, sizeof(double) * SPK_CLOSURE_NPARAM);
    double L = 0.0;
    for (size_t s = 0; s < n; s++) {
        double f[NF], S[5], J[3], tT[5], tE[3], Sf[5], Jf[3];
        for (int r = 0; r < 5; r++) Sf[r] = X[(SPK_CLOSURE_ROW_SF + r) * stride + s];
        for (int r = 0; r < 3; r++) Jf[r] = X[(SPK_CLOSURE_ROW_JF + r) * stride + s];
        for (int r = 0; r < NF; r++) f[r] = X[(SPK_CLOSURE_ROW_FEAT + r) * stride + s];
        for (int r = 0; r < 5; r++) S[r] = X[(SPK_CLOSURE_ROW_S + r) * stride + s];
        for (int r = 0; r < 3; r++) J[r] = X[(SPK_CLOSURE_ROW_J + r) * stride + s];
        const double scale = X[SPK_CLOSURE_ROW_SCALE * stride + s];
        for (int r = 0; r < 5; r++) tT[r] = X[(SPK_CLOSURE_ROW_TT + r) * stride + s];
        for (int r = 0; r < 3; r++) tE[r] = X[(SPK_CLOSURE_ROW_TE + r) * stride + s];
        double h1[NH], h2[NH], o[NO];
        forward(P, f, h1, h2, o);
        const double nu = scale * softplus(o[0]), eta = scale * softplus(o[1]);
        /* stress error in the 5-channel basis; zz = -(xx + yy) */
        double e[5];
        for (int r = 0; r < 5; r++) e[r] = -2.0 * nu * S[r] - tT[r];
        const double ezz = -(e[0] + e[3]);
        const double fro = e[0] * e[0] + e[3] * e[3] + ezz * ezz + 2.0 * (e[1] * e[1] + e[2] * e[2] + e[4] * e[4]);
        double eE[3], emf = 0.0;
        for (int r = 0; r < 3; r++) { eE[r] = -eta * J[r] - tE[r]; emf += eE[r] * eE[r]; }
        /* dissipation matching: P = 2 nu S:Sf + eta J.Jf against -tT:Sf - tE.Jf */
        const double SSf = S[0] * Sf[0] + S[3] * Sf[3] + (S[0] + S[3]) * (Sf[0] + Sf[3]) +
                           2.0 * (S[1] * Sf[1] + S[2] * Sf[2] + S[4] * Sf[4]);
        const double TSf = tT[0] * Sf[0] + tT[3] * Sf[3] + (tT[0] + tT[3]) * (Sf[0] + Sf[3]) +
                           2.0 * (tT[1] * Sf[1] + tT[2] * Sf[2] + tT[4] * Sf[4]);
        double JJf = 0.0, EJf = 0.0;
        for (int r = 0; r < 3; r++) { JJf += J[r] * Jf[r]; EJf += tE[r] * Jf[r]; }
        const double dP = (2.0 * nu * SSf + eta * JJf) - (-TSf - EJf);
        L += w[0] * fro + w[1] * emf + w[2] * dP * dP;
        /* d fro / d e: zz enters through e0 and e3 */
        double ge[5];
        ge[0] = 2.0 * e[0] - 2.0 * ezz;
        ge[3] = 2.0 * e[3] - 2.0 * ezz;
        ge[1] = 4.0 * e[1]; ge[2] = 4.0 * e[2]; ge[4] = 4.0 * e[4];
        double dnu = 0.0, deta = 0.0;
        for (int r = 0; r < 5; r++) dnu += w[0] * ge[r] * (-2.0 * S[r]);
        for (int r = 0; r < 3; r++) deta += w[1] * 2.0 * eE[r] * (-J[r]);
        dnu += w[2] * 2.0 * dP * 2.0 * SSf;
        deta += w[2] * 2.0 * dP * JJf;
        double d3[NO];
        d3[0] = dnu * scale * sigmoid(o[0]);
        d3[1] = deta * scale * sigmoid(o[1]);
        double d2[NH], d1[NH];
        for (int i = 0; i < NH; i++) {
            double a = 0.0;
            for (int j = 0; j < NO; j++) a += P[OW3 + j * NH + i] * d3[j];
            d2[i] = a * (1.0 - h2[i] * h2[i]);
        }
        for (int i = 0; i < NH; i++) {
            double a = 0.0;
            for (int j = 0; j < NH; j++) a += P[OW2 + j * NH + i] * d2[j];
            d1[i] = a * (1.0 - h1[i] * h1[i]);
        }
        for (int j = 0; j < NO; j++) {
            grad[OB3 + j] += d3[j];
            for (int i = 0; i < NH; i++) grad[OW3 + j * NH + i] += d3[j] * h2[i];
        }
        for (int j = 0; j < NH; j++) {
            grad[OB2 + j] += d2[j];
            for (int i = 0; i < NH; i++) grad[OW2 + j * NH + i] += d2[j] * h1[i];
        }
        for (int j = 0; j < NH; j++) {
            grad[OB1 + j] += d1[j];
            for (int i = 0; i < NF; i++) grad[OW1 + j * NF + i] += d1[j] * f[i];
        }
    }
    const double inv = n > 0 ? 1.0 / (double)n : 0.0;
    for (int p = 0; p < SPK_CLOSURE_NPARAM; p++) grad[p] *= inv;
    *loss = L * inv;
}

void orc_closure_adam(double* P, const double* g, double* m, double* v, int t, double lr) {
    const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    const double c1 = 1.0 - pow(b1, t), c2 = 1.0 - pow(b2, t);
    for (int p = 0; p < SPK_CLOSURE_NPARAM; p++) {
        m[p] = b1 * m[p] + (1.0 - b1) * g[p];
        v[p] = b2 * v[p] + (1.0 - b2) * g[p] * g[p];
        P[p] -= lr * (m[p] / c1) / (sqrt(v[p] / c2) + eps);
    }
}
