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
#include <stdint.h>
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

/* ---- variant 3: the tensor network (include/spooky_b200.h, SPK_CLOSURE3_*).
 * Every operand the CUDA kernels feed to a BF16 tensor-core product is
 * rounded here at the same place (weights, layer inputs, back-propagated
 * errors); sums run in FP64 (the kernels: FP32).  orc_closure3_set_rounding(0)
 * drops the roundings, which makes the loss smooth in the parameters for a
 * finite-difference check of the gradient formulas. */
enum { N3I = SPK_CLOSURE3_NIN, N3H = SPK_CLOSURE3_HIDDEN, N3O = SPK_CLOSURE3_NOUT };
enum {
    Q1 = 0, QB1 = Q1 + N3H * N3I, Q2 = QB1 + N3H, QB2 = Q2 + N3H * N3H, Q3 = QB2 + N3H,
    QB3 = Q3 + N3H * N3H, Q4 = QB3 + N3H, QB4 = Q4 + N3O * N3H, QN = QB4 + N3O
};

static int g_bf16 = 1;
void orc_closure3_set_rounding(int on) { g_bf16 = on; }

/* x to FP32, then to BF16 with round-to-nearest-even on the 16 dropped bits */
static double bf(double x) {
    if (!g_bf16) return x;
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x7fffu + ((u >> 16) & 1u);
        u &= 0xffff0000u;
    }
    memcpy(&f, &u, 4);
    return (double)f;
}

/* the network on x[18]: rounded input xb, rounded activations h1..h3, outputs o[12] */
static void fwd3(const double* P, const double* x, double* xb, double* h1, double* h2, double* h3, double* o) {
    for (int i = 0; i < N3I; i++) xb[i] = bf(x[i]);
    for (int j = 0; j < N3H; j++) {
        double a = P[QB1 + j];
        for (int i = 0; i < N3I; i++) a += bf(P[Q1 + j * N3I + i]) * xb[i];
        h1[j] = bf(tanh(a));
    }
    for (int j = 0; j < N3H; j++) {
        double a = P[QB2 + j];
        for (int i = 0; i < N3H; i++) a += bf(P[Q2 + j * N3H + i]) * h1[i];
        h2[j] = bf(tanh(a));
    }
    for (int j = 0; j < N3H; j++) {
        double a = P[QB3 + j];
        for (int i = 0; i < N3H; i++) a += bf(P[Q3 + j * N3H + i]) * h2[i];
        h3[j] = bf(tanh(a));
    }
    for (int j = 0; j < N3O; j++) {
        double a = P[QB4 + j];
        for (int i = 0; i < N3H; i++) a += bf(P[Q4 + j * N3H + i]) * h3[i];
        o[j] = a;
    }
}

/* the model's traceless stress dT[5] and EMF dE[3] from s = Delta^2 n^2 o */
static void tensor_terms(const double* s, double* dT, double* dE) {
    const double tr = (s[0] + s[3] + s[5]) / 3.0;
    dT[0] = s[0] - tr; dT[1] = s[1]; dT[2] = s[2]; dT[3] = s[3] - tr; dT[4] = s[4];
    /* M_xy M_xz M_yx M_yz M_zx M_zy = s6 .. s11 */
    dE[0] = 0.5 * (s[9] - s[11]);
    dE[1] = 0.5 * (s[10] - s[7]);
    dE[2] = 0.5 * (s[6] - s[8]);
}

void orc_closure3_mlp(const double* params, const double* x, double* o) {
    double xb[N3I], h1[N3H], h2[N3H], h3[N3H];
    fwd3(params, x, xb, h1, h2, h3, o);
}

double orc_closure3_terms(const double* P, double delta2, const double* A, const double* G, int mhd, double* tau,
                          double* e, double* nu_eff, double* eta_eff) {
    double f[8], S5[5], J3[3], x[N3I], o[N3O], s[N3O], dT[5], dE[3];
    const double n = orc_closure_features(A, G, f, S5, J3);
    for (int i = 0; i < 9; i++) { x[i] = A[i] / n; x[9 + i] = G[i] / n; }
    orc_closure3_mlp(P, x, o);
    for (int i = 0; i < N3O; i++) s[i] = delta2 * n * n * o[i];
    tensor_terms(s, dT, dE);
    if (!mhd) dE[0] = dE[1] = dE[2] = 0.0;
    const double Szz = A[8], dTzz = -(dT[0] + dT[3]);
    const double TS = dT[0] * S5[0] + dT[3] * S5[3] + dTzz * Szz + 2.0 * (dT[1] * S5[1] + dT[2] * S5[2] + dT[4] * S5[4]);
    const double T2 = dT[0] * dT[0] + dT[3] * dT[3] + dTzz * dTzz + 2.0 * (dT[1] * dT[1] + dT[2] * dT[2] + dT[4] * dT[4]);
    const double S2 = S5[0] * S5[0] + S5[3] * S5[3] + Szz * Szz + 2.0 * (S5[1] * S5[1] + S5[2] * S5[2] + S5[4] * S5[4]);
    double EJ = 0.0, E2 = 0.0, J2 = 0.0;
    for (int k = 0; k < 3; k++) { EJ += dE[k] * J3[k]; E2 += dE[k] * dE[k]; J2 += J3[k] * J3[k]; }
    const double Pt = -TS - EJ, Pm = sqrt(T2) * sqrt(S2) + sqrt(E2) * sqrt(J2);
    double r = Pt / (0.1 * Pm + 1e-30);
    r = r < 0.0 ? 0.0 : (r > 1.0 ? 1.0 : r);
    for (int k = 0; k < 5; k++) tau[k] = r * dT[k];
    for (int k = 0; k < 3; k++) e[k] = r * dE[k];
    *nu_eff = r * sqrt(T2) / (2.0 * n);
    *eta_eff = mhd ? r * sqrt(E2) / n : 0.0;
    return n;
}

void orc_closure3_loss_grad(const double* X, size_t n, size_t stride, const double* P, const double* w, double* grad,
                            double* loss) {
    memset(grad, 0, sizeof(double) * QN);
    double L = 0.0;
    double W4b[N3O * N3H], W3b[N3H * N3H], W2b[N3H * N3H];
    for (int i = 0; i < N3O * N3H; i++) W4b[i] = bf(P[Q4 + i]);
    for (int i = 0; i < N3H * N3H; i++) { W3b[i] = bf(P[Q3 + i]); W2b[i] = bf(P[Q2 + i]); }
    for (size_t q = 0; q < n; q++) {
        double A[9], G[9], f[8], S5[5], J3[3], x[N3I], xb[N3I], h1[N3H], h2[N3H], h3[N3H], o[N3O];
        double tT[5], tE[3], Sf[5], Jf[3], s[N3O], dT[5], dE[3];
        for (int r = 0; r < 9; r++) {
            A[r] = X[(SPK_CLOSURE_ROW_A + r) * stride + q];
            G[r] = X[(SPK_CLOSURE_ROW_G + r) * stride + q];
        }
        for (int r = 0; r < 5; r++) { tT[r] = X[(SPK_CLOSURE_ROW_TT + r) * stride + q]; Sf[r] = X[(SPK_CLOSURE_ROW_SF + r) * stride + q]; }
        for (int r = 0; r < 3; r++) { tE[r] = X[(SPK_CLOSURE_ROW_TE + r) * stride + q]; Jf[r] = X[(SPK_CLOSURE_ROW_JF + r) * stride + q]; }
        const double nn = orc_closure_features(A, G, f, S5, J3);
        const double sc = X[SPK_CLOSURE_ROW_SCALE * stride + q] * nn;   /* Delta^2 n^2 */
        for (int i = 0; i < 9; i++) { x[i] = A[i] / nn; x[9 + i] = G[i] / nn; }
        fwd3(P, x, xb, h1, h2, h3, o);
        for (int i = 0; i < N3O; i++) s[i] = sc * o[i];
        tensor_terms(s, dT, dE);
        double e[5], eE[3];
        for (int r = 0; r < 5; r++) e[r] = dT[r] - tT[r];
        for (int r = 0; r < 3; r++) eE[r] = dE[r] - tE[r];
        const double ezz = -(e[0] + e[3]), Sfzz = -(Sf[0] + Sf[3]);
        const double fro = e[0] * e[0] + e[3] * e[3] + ezz * ezz + 2.0 * (e[1] * e[1] + e[2] * e[2] + e[4] * e[4]);
        double emf = 0.0, eJ = 0.0;
        for (int r = 0; r < 3; r++) { emf += eE[r] * eE[r]; eJ += eE[r] * Jf[r]; }
        /* transfer error: -(dT - tT):Sf - (dE - tE).Jf */
        const double dP = -(e[0] * Sf[0] + e[3] * Sf[3] + ezz * Sfzz + 2.0 * (e[1] * Sf[1] + e[2] * Sf[2] + e[4] * Sf[4])) - eJ;
        L += w[0] * fro + w[1] * emf + w[2] * dP * dP;
        /* d loss / d e (e5 independent, ezz through e0 and e3), d loss / d eE */
        double g5[5], gE[3];
        g5[0] = w[0] * (2.0 * e[0] - 2.0 * ezz) + w[2] * 2.0 * dP * -(Sf[0] - Sfzz);
        g5[3] = w[0] * (2.0 * e[3] - 2.0 * ezz) + w[2] * 2.0 * dP * -(Sf[3] - Sfzz);
        g5[1] = w[0] * 4.0 * e[1] + w[2] * 2.0 * dP * -2.0 * Sf[1];
        g5[2] = w[0] * 4.0 * e[2] + w[2] * 2.0 * dP * -2.0 * Sf[2];
        g5[4] = w[0] * 4.0 * e[4] + w[2] * 2.0 * dP * -2.0 * Sf[4];
        for (int r = 0; r < 3; r++) gE[r] = w[1] * 2.0 * eE[r] + w[2] * 2.0 * dP * -Jf[r];
        /* through dT(s), dE(s) and s = sc o */
        double gs[N3O], d4[N3O], d3[N3H], d2[N3H], d1[N3H];
        gs[0] = (2.0 * g5[0] - g5[3]) / 3.0;
        gs[3] = (2.0 * g5[3] - g5[0]) / 3.0;
        gs[5] = -(g5[0] + g5[3]) / 3.0;
        gs[1] = g5[1]; gs[2] = g5[2]; gs[4] = g5[4];
        gs[9] = 0.5 * gE[0]; gs[11] = -0.5 * gE[0];
        gs[10] = 0.5 * gE[1]; gs[7] = -0.5 * gE[1];
        gs[6] = 0.5 * gE[2]; gs[8] = -0.5 * gE[2];
        for (int j = 0; j < N3O; j++) d4[j] = bf(sc * gs[j]);
        for (int i = 0; i < N3H; i++) {
            double a = 0.0;
            for (int j = 0; j < N3O; j++) a += W4b[j * N3H + i] * d4[j];
            d3[i] = bf(a * (1.0 - h3[i] * h3[i]));
        }
        for (int i = 0; i < N3H; i++) {
            double a = 0.0;
            for (int j = 0; j < N3H; j++) a += W3b[j * N3H + i] * d3[j];
            d2[i] = bf(a * (1.0 - h2[i] * h2[i]));
        }
        for (int i = 0; i < N3H; i++) {
            double a = 0.0;
            for (int j = 0; j < N3H; j++) a += W2b[j * N3H + i] * d2[j];
            d1[i] = bf(a * (1.0 - h1[i] * h1[i]));
        }
        for (int j = 0; j < N3O; j++) {
            grad[QB4 + j] += d4[j];
            for (int i = 0; i < N3H; i++) grad[Q4 + j * N3H + i] += d4[j] * h3[i];
        }
        for (int j = 0; j < N3H; j++) {
            grad[QB3 + j] += d3[j];
            grad[QB2 + j] += d2[j];
            grad[QB1 + j] += d1[j];
            for (int i = 0; i < N3H; i++) {
                grad[Q3 + j * N3H + i] += d3[j] * h2[i];
                grad[Q2 + j * N3H + i] += d2[j] * h1[i];
            }
            for (int i = 0; i < N3I; i++) grad[Q1 + j * N3I + i] += d1[j] * xb[i];
        }
    }
    const double inv = n > 0 ? 1.0 / (double)n : 0.0;
    for (int p = 0; p < QN; p++) grad[p] *= inv;
    *loss = L * inv;
}

void orc_closure_adam_n(double* P, const double* g, double* m, double* v, int t, double lr, int np) {
    const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    const double c1 = 1.0 - pow(b1, t), c2 = 1.0 - pow(b2, t);
    for (int p = 0; p < np; p++) {
        m[p] = b1 * m[p] + (1.0 - b1) * g[p];
        v[p] = b2 * v[p] + (1.0 - b2) * g[p] * g[p];
        P[p] -= lr * (m[p] / c1) / (sqrt(v[p] / c2) + eps);
    }
}
