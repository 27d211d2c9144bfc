// spk_closure.cuh -- the learned subgrid closure's pointwise math on sm_100a:
// the rotation-invariant features of the velocity and field gradients and
// the MLP that maps them to an eddy viscosity and an eddy resistivity
// (definition in include/spooky_b200.h, SPK_CLOSURE_*).  Used inside the z
// pass (fused inference, FP32) and by the sample kernels.
#pragma once

namespace spk {

enum { CL_NF = 8, CL_NH = 32, CL_NO = 2 };
// parameter offsets: W1[32][8] b1[32] W2[32][32] b2[32] W3[2][32] b3[2]
enum {
    CL_W1 = 0,
    CL_B1 = CL_W1 + CL_NH * CL_NF,
    CL_W2 = CL_B1 + CL_NH,
    CL_B2 = CL_W2 + CL_NH * CL_NH,
    CL_W3 = CL_B2 + CL_NH,
    CL_B3 = CL_W3 + CL_NO * CL_NH,
    CL_NP = CL_B3 + CL_NO
};

// A[3*i + j] = du_i/dx_j, G likewise for B.  Writes the features f[8], the
// strain S (xx xy xz yy yz) and the current J; returns n.
template <typename R>
__host__ __device__ __forceinline__ R closure_features(const R* A, const R* G, R* f, R* S5, R* J3) {
    const R h = (R)0.5;
    const R S00 = A[0], S11 = A[4], S22 = A[8];
    const R S01 = h * (A[1] + A[3]), S02 = h * (A[2] + A[6]), S12 = h * (A[5] + A[7]);
    const R B00 = G[0], B11 = G[4], B22 = G[8];
    const R B01 = h * (G[1] + G[3]), B02 = h * (G[2] + G[6]), B12 = h * (G[5] + G[7]);
    const R w0 = A[7] - A[5], w1 = A[2] - A[6], w2 = A[3] - A[1];   // curl u
    const R j0 = G[7] - G[5], j1 = G[2] - G[6], j2 = G[3] - G[1];   // curl B
    const R s2 = S00 * S00 + S11 * S11 + S22 * S22 + (R)2 * (S01 * S01 + S02 * S02 + S12 * S12);
    const R b2 = B00 * B00 + B11 * B11 + B22 * B22 + (R)2 * (B01 * B01 + B02 * B02 + B12 * B12);
    const R ww = h * (w0 * w0 + w1 * w1 + w2 * w2);
    const R jj = h * (j0 * j0 + j1 * j1 + j2 * j2);
    // tr(S^3) of a symmetric S
    const R tr3 = S00 * S00 * S00 + S11 * S11 * S11 + S22 * S22 * S22 +
                  (R)3 * (S01 * S01 * (S00 + S11) + S02 * S02 * (S00 + S22) + S12 * S12 * (S11 + S22)) +
                  (R)6 * S01 * S02 * S12;
    auto quad = [&](R x, R y, R z) {   // v.S.v
        return S00 * x * x + S11 * y * y + S22 * z * z + (R)2 * (S01 * x * y + S02 * x * z + S12 * y * z);
    };
    const R wsw = quad(w0, w1, w2), jsj = quad(j0, j1, j2);
    const R wj = w0 * j0 + w1 * j1 + w2 * j2;
    const R n2 = s2 + ww + b2 + jj + (R)1e-30;
    const R n = sqrt(n2);
    const R i2 = (R)1 / n2, i3 = i2 / n;
    f[0] = s2 * i2;
    f[1] = ww * i2;
    f[2] = b2 * i2;
    f[3] = jj * i2;
    f[4] = tr3 * i3;
    f[5] = wsw * i3;
    f[6] = jsj * i3;
    f[7] = wj * wj * (R)0.25 * i2 * i2;
    S5[0] = S00; S5[1] = S01; S5[2] = S02; S5[3] = S11; S5[4] = S12;
    J3[0] = j0; J3[1] = j1; J3[2] = j2;
    return n;
}

__device__ __forceinline__ float closure_softplus(float x) { return x > 30.f ? x : log1pf(expf(x)); }

// MLP outputs o[2] for features f (parameters in shared memory: every lane
// of a warp reads the same word, a broadcast).
__device__ __forceinline__ void closure_mlp(const float* __restrict__ P, const float* f, float* o) {
    float h1[CL_NH];
#pragma unroll
    for (int j = 0; j < CL_NH; j++) {
        float a = P[CL_B1 + j];
#pragma unroll
        for (int i = 0; i < CL_NF; i++) a = fmaf(P[CL_W1 + j * CL_NF + i], f[i], a);
        h1[j] = tanhf(a);
    }
    float o0 = P[CL_B3], o1 = P[CL_B3 + 1];
#pragma unroll 4
    for (int j = 0; j < CL_NH; j++) {
        float a = P[CL_B2 + j];
#pragma unroll
        for (int i = 0; i < CL_NH; i++) a = fmaf(P[CL_W2 + j * CL_NH + i], h1[i], a);
        const float h2 = tanhf(a);
        o0 = fmaf(P[CL_W3 + j], h2, o0);
        o1 = fmaf(P[CL_W3 + CL_NH + j], h2, o1);
    }
    o[0] = o0;
    o[1] = o1;
}

// Closure terms at one point: tau[5] = -2 nu_t S, e[3] = -eta_t J; returns
// nu_t and eta_t through nu, eta.
__device__ __forceinline__ void closure_point(const float* __restrict__ P, float delta2, const float* A, const float* G,
                                              float* tau, float* e, float* nu, float* eta) {
    float f[CL_NF], S5[5], J3[3], o[2];
    const float n = closure_features<float>(A, G, f, S5, J3);
    closure_mlp(P, f, o);
    const float sc = delta2 * n;
    const float vn = sc * closure_softplus(o[0]), ve = sc * closure_softplus(o[1]);
#pragma unroll
    for (int r = 0; r < 5; r++) tau[r] = -2.f * vn * S5[r];
#pragma unroll
    for (int r = 0; r < 3; r++) e[r] = -ve * J3[r];
    *nu = vn;
    *eta = ve;
}

}  // namespace spk
