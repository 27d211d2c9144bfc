// spk_closure.cu -- training and data-preparation kernels of the learned
// subgrid closure (definition in include/spooky_b200.h, SPK_CLOSURE_*).
//
// Training: one thread per sample runs the forward pass and the backward
// pass of the loss through the MLP in registers and parks the activations
// and back-propagated errors of its 128-sample chunk in shared memory; the
// CTA then forms the weight gradients of the chunk (one parameter per thread
// and round, a fixed-order sum over the chunk) and keeps them in registers
// across its chunks.  A second kernel sums the per-CTA partials in FP64 in a
// fixed order, so the gradient is deterministic.  Adam is one thread per
// parameter.
#include "spk_closure.cuh"
#include "spk_closure3.cuh"

namespace spk {

#define CL_CHUNK 128
#define CL_LDS (CL_CHUNK + 1)                 // padded row: rows i, i+1 start in different banks
#define CL_ROWS (CL_NF + 4 * CL_NH + CL_NO)   // x, h1, h2, d1, d2, d3 per sample
#define CL_PPT ((CL_NP + CL_CHUNK - 1) / CL_CHUNK)
#define CL_MAXBLK (148 * 2)

struct TrainArgs {
    const float* X;          // sample rows
    size_t n, stride;        // samples, floats between rows
    size_t m;                // samples in this evaluation (n: full batch)
    int minibatch;           // 1: sample r -> (a * ((base + r) mod n) + c) mod n
    unsigned long long a, c, base;
    const float* params;
    float w0, w1, w2;        // loss weights (stress, EMF, energy transfer)
    float* partial;          // [gridDim.x][CL_NP + 1] (last: loss)
};

__global__ void __launch_bounds__(CL_CHUNK) k_closure_grad(const __grid_constant__ TrainArgs a) {
    extern __shared__ __align__(16) float cl_smem[];
    float* P = cl_smem;                           // parameters
    float* act = cl_smem + ((CL_NP + 3) & ~3);    // [CL_ROWS][CL_LDS]
    const int tid = threadIdx.x;
    for (int i = tid; i < CL_NP; i += CL_CHUNK) P[i] = a.params[i];
    float acc[CL_PPT];
#pragma unroll
    for (int k = 0; k < CL_PPT; k++) acc[k] = 0.f;
    float lsum = 0.f;
    float* sx = act;
    float* sh1 = sx + CL_NF * CL_LDS;
    float* sh2 = sh1 + CL_NH * CL_LDS;
    float* sd1 = sh2 + CL_NH * CL_LDS;
    float* sd2 = sd1 + CL_NH * CL_LDS;
    float* sd3 = sd2 + CL_NH * CL_LDS;
    const size_t nch = (a.m + CL_CHUNK - 1) / CL_CHUNK;
    __syncthreads();
    for (size_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const size_t r = ch * CL_CHUNK + tid;
        const bool valid = r < a.m;
        float f[CL_NF], S[5], J[3], tT[5], tE[3], Sf[5], Jf[3], scale = 0.f;
        if (valid) {
            size_t s = r;
            if (a.minibatch) s = (size_t)((a.a * ((a.base + r) % a.n) + a.c) % a.n);
            const float* X = a.X + s;
#pragma unroll
            for (int i = 0; i < CL_NF; i++) f[i] = X[(size_t)(SPK_CLOSURE_ROW_FEAT + i) * a.stride];
#pragma unroll
            for (int i = 0; i < 5; i++) S[i] = X[(size_t)(SPK_CLOSURE_ROW_S + i) * a.stride];
#pragma unroll
            for (int i = 0; i < 3; i++) J[i] = X[(size_t)(SPK_CLOSURE_ROW_J + i) * a.stride];
            scale = X[(size_t)SPK_CLOSURE_ROW_SCALE * a.stride];
#pragma unroll
            for (int i = 0; i < 5; i++) tT[i] = X[(size_t)(SPK_CLOSURE_ROW_TT + i) * a.stride];
#pragma unroll
            for (int i = 0; i < 3; i++) tE[i] = X[(size_t)(SPK_CLOSURE_ROW_TE + i) * a.stride];
#pragma unroll
            for (int i = 0; i < 5; i++) Sf[i] = X[(size_t)(SPK_CLOSURE_ROW_SF + i) * a.stride];
#pragma unroll
            for (int i = 0; i < 3; i++) Jf[i] = X[(size_t)(SPK_CLOSURE_ROW_JF + i) * a.stride];
        } else {
#pragma unroll
            for (int i = 0; i < CL_NF; i++) f[i] = 0.f;
#pragma unroll
            for (int i = 0; i < 5; i++) { S[i] = 0.f; tT[i] = 0.f; Sf[i] = 0.f; }
#pragma unroll
            for (int i = 0; i < 3; i++) { J[i] = 0.f; tE[i] = 0.f; Jf[i] = 0.f; }
        }
        // forward
        float h1[CL_NH], h2[CL_NH];
#pragma unroll
        for (int j = 0; j < CL_NH; j++) {
            float v = P[CL_B1 + j];
#pragma unroll
            for (int i = 0; i < CL_NF; i++) v = fmaf(P[CL_W1 + j * CL_NF + i], f[i], v);
            h1[j] = tanhf(v);
        }
        float o0 = P[CL_B3], o1 = P[CL_B3 + 1];
#pragma unroll 4
        for (int j = 0; j < CL_NH; j++) {
            float v = P[CL_B2 + j];
#pragma unroll
            for (int i = 0; i < CL_NH; i++) v = fmaf(P[CL_W2 + j * CL_NH + i], h1[i], v);
            h2[j] = tanhf(v);
            o0 = fmaf(P[CL_W3 + j], h2[j], o0);
            o1 = fmaf(P[CL_W3 + CL_NH + j], h2[j], o1);
        }
        const float nu = scale * closure_softplus(o0), eta = scale * closure_softplus(o1);
        // loss and its derivative with respect to nu_t and eta_t
        float e[5];
#pragma unroll
        for (int i = 0; i < 5; i++) e[i] = -2.f * nu * S[i] - tT[i];
        const float ezz = -(e[0] + e[3]);
        const float fro = e[0] * e[0] + e[3] * e[3] + ezz * ezz + 2.f * (e[1] * e[1] + e[2] * e[2] + e[4] * e[4]);
        float eE[3], emf = 0.f;
#pragma unroll
        for (int i = 0; i < 3; i++) { eE[i] = -eta * J[i] - tE[i]; emf += eE[i] * eE[i]; }
        // energy transfer into the subgrid scales: model 2 nu S:Sf + eta J.Jf
        // against the true -T:Sf - E.Jf (Sf, Jf of the whole resolved field)
        const float SSf = S[0] * Sf[0] + S[3] * Sf[3] + (S[0] + S[3]) * (Sf[0] + Sf[3]) +
                          2.f * (S[1] * Sf[1] + S[2] * Sf[2] + S[4] * Sf[4]);
        const float TSf = tT[0] * Sf[0] + tT[3] * Sf[3] + (tT[0] + tT[3]) * (Sf[0] + Sf[3]) +
                          2.f * (tT[1] * Sf[1] + tT[2] * Sf[2] + tT[4] * Sf[4]);
        const float JJf = J[0] * Jf[0] + J[1] * Jf[1] + J[2] * Jf[2];
        const float EJf = tE[0] * Jf[0] + tE[1] * Jf[1] + tE[2] * Jf[2];
        const float dP = 2.f * nu * SSf + eta * JJf + TSf + EJf;
        if (valid) lsum += a.w0 * fro + a.w1 * emf + a.w2 * dP * dP;
        const float ge0 = 2.f * e[0] - 2.f * ezz, ge3 = 2.f * e[3] - 2.f * ezz;
        const float dnu = a.w0 * -2.f * (ge0 * S[0] + ge3 * S[3] + 4.f * (e[1] * S[1] + e[2] * S[2] + e[4] * S[4])) +
                          a.w2 * 4.f * dP * SSf;
        float deta = a.w2 * 2.f * dP * JJf;
#pragma unroll
        for (int i = 0; i < 3; i++) deta += a.w1 * 2.f * eE[i] * -J[i];
        const float d30 = valid ? dnu * scale / (1.f + expf(-o0)) : 0.f;
        const float d31 = valid ? deta * scale / (1.f + expf(-o1)) : 0.f;
        // backward through the hidden layers; activations and errors to shared memory
        float d2[CL_NH];
#pragma unroll
        for (int i = 0; i < CL_NH; i++) {
            const float v = P[CL_W3 + i] * d30 + P[CL_W3 + CL_NH + i] * d31;
            d2[i] = v * (1.f - h2[i] * h2[i]);
        }
        __syncthreads();   // the previous chunk's gradient sums have read the tile
#pragma unroll
        for (int i = 0; i < CL_NF; i++) sx[i * CL_LDS + tid] = f[i];
#pragma unroll
        for (int i = 0; i < CL_NH; i++) {
            sh1[i * CL_LDS + tid] = h1[i];
            sh2[i * CL_LDS + tid] = h2[i];
            sd2[i * CL_LDS + tid] = d2[i];
        }
        sd3[tid] = d30;
        sd3[CL_LDS + tid] = d31;
#pragma unroll 4
        for (int i = 0; i < CL_NH; i++) {
            float v = 0.f;
#pragma unroll
            for (int j = 0; j < CL_NH; j++) v = fmaf(P[CL_W2 + j * CL_NH + i], d2[j], v);
            sd1[i * CL_LDS + tid] = v * (1.f - h1[i] * h1[i]);
        }
        __syncthreads();
        // weight gradients of the chunk: parameter p = tid + k * CL_CHUNK
#pragma unroll
        for (int k = 0; k < CL_PPT; k++) {
            const int p = tid + k * CL_CHUNK;
            if (p >= CL_NP) break;
            const float* dr;
            const float* ar = nullptr;
            if (p < CL_B1) { dr = sd1 + (p / CL_NF) * CL_LDS; ar = sx + (p % CL_NF) * CL_LDS; }
            else if (p < CL_W2) { dr = sd1 + (p - CL_B1) * CL_LDS; }
            else if (p < CL_B2) { const int q = p - CL_W2; dr = sd2 + (q / CL_NH) * CL_LDS; ar = sh1 + (q % CL_NH) * CL_LDS; }
            else if (p < CL_W3) { dr = sd2 + (p - CL_B2) * CL_LDS; }
            else if (p < CL_B3) { const int q = p - CL_W3; dr = sd3 + (q / CL_NH) * CL_LDS; ar = sh2 + (q % CL_NH) * CL_LDS; }
            else { dr = sd3 + (p - CL_B3) * CL_LDS; }
            float s = 0.f;
            if (ar) {
                for (int t = 0; t < CL_CHUNK; t++) s = fmaf(dr[t], ar[t], s);
            } else {
                for (int t = 0; t < CL_CHUNK; t++) s += dr[t];
            }
            acc[k] += s;
        }
    }
    float* out = a.partial + (size_t)blockIdx.x * (CL_NP + 1);
#pragma unroll
    for (int k = 0; k < CL_PPT; k++) {
        const int p = tid + k * CL_CHUNK;
        if (p < CL_NP) out[p] = acc[k];
    }
    // block sum of the loss in a fixed order
    __syncthreads();
    act[tid] = lsum;
    __syncthreads();
    if (tid == 0) {
        float s = 0.f;
        for (int t = 0; t < CL_CHUNK; t++) s += act[t];
        out[CL_NP] = s;
    }
}

// grad[p] = sum over CTAs of partial[b][p] / m (FP64, fixed order); the loss
// goes to loss_out.
__global__ void k_closure_reduce(const float* partial, int nblk, double inv_m, float* grad, float* loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > CL_NP) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += (double)partial[(size_t)b * (CL_NP + 1) + p];
    if (p < CL_NP) grad[p] = (float)(s * inv_m);
    else if (loss_out) *loss_out = (float)(s * inv_m);
}

// One Adam step, t >= 1 (Kingma & Ba 2015; beta1 0.9, beta2 0.999, eps 1e-8).
__global__ void k_closure_adam(float* params, const float* grad, float* m, float* v, int t, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= CL_NP) return;
    const double b1 = 0.9, b2 = 0.999;
    const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
    const float g = grad[p];
    const float mm = (float)(b1 * m[p] + (1.0 - b1) * g);
    const float vv = (float)(b2 * v[p] + (1.0 - b2) * (double)g * g);
    m[p] = mm;
    v[p] = vv;
    params[p] -= (float)(lr * (mm / c1) / (sqrt(vv / c2) + 1e-8));
}

// ---------------------------------------------------------------------------
// data preparation
// ---------------------------------------------------------------------------
// Sharp spectral filter: the coarse grid's kept modes of fine-grid spectra
// (scaled by the point-count ratio), zero elsewhere; nch channels.
struct TruncArgs {
    const double2* src; double2* dst;
    int nch;
    int fnx, fny, fnzh;           // fine grid
    int cnx, cny, cnzh;           // coarse grid
    const double *mx, *my, *mz;   // coarse mask factors
    double scale;
};
__global__ void k_truncate(const __grid_constant__ TruncArgs a) {
    const size_t ncc = (size_t)a.cnx * a.cny * a.cnzh, ncf = (size_t)a.fnx * a.fny * a.fnzh;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < ncc * a.nch; gi += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(gi / ncc);
        const size_t id = gi - (size_t)ch * ncc;
        const int k = (int)(id % a.cnzh);
        const size_t rr = id / a.cnzh;
        const int j = (int)(rr % a.cny), i = (int)(rr / a.cny);
        double2 v = make_double2(0.0, 0.0);
        if (a.mx[i] * a.my[j] * a.mz[k] != 0.0) {
            const int ix = i < a.cnx / 2 ? i : i - a.cnx, iy = j < a.cny / 2 ? j : j - a.cny;
            const int fi = ix >= 0 ? ix : ix + a.fnx, fj = iy >= 0 ? iy : iy + a.fny;
            const double2 s = a.src[(size_t)ch * ncf + (size_t)k + (size_t)a.fnzh * ((size_t)fj + (size_t)fi * a.fny)];
            v = make_double2(a.scale * s.x, a.scale * s.y);
        }
        a.dst[gi] = v;
    }
}

// y -= x over n complex values
__global__ void k_sub(double2* y, const double2* x, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = make_double2(y[i].x - x[i].x, y[i].y - x[i].y);
}

// Spectral gradients: out[9 b + 3 i + j] = i k_j U_{field(b, i)} (b = 0: u, 1: B);
// hp_k2 > 0: only modes with |k|^2 > hp_k2 (the closure's variant 2).
__global__ void k_gradients(const DevGrid g, const double2* U, int VEL, int MAG, int nb, double hp_k2, double2* out) {
    const size_t nc = g.nc;
    for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < nc; id += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(id % g.nzh);
        const size_t rr = id / g.nzh;
        const int j = (int)(rr % g.ny), i = (int)(rr / g.ny);
        const double kv[3] = {g.kx[i], g.ky[j], g.kz[k]};
        const bool keep = !(hp_k2 > 0.0) || kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2] > hp_k2;
        for (int b = 0; b < nb; b++)
            for (int c = 0; c < 3; c++) {
                const double2 x = U[(size_t)((b ? MAG : VEL) + c) * nc + id];
                for (int d = 0; d < 3; d++)
                    out[(size_t)(9 * b + 3 * c + d) * nc + id] =
                        keep ? make_double2(-kv[d] * x.y, kv[d] * x.x) : make_double2(0.0, 0.0);
            }
    }
}

// Sample rows from the real-space gradients Rg[18][nr] of the model's input,
// the whole field's gradients Rgf[18][nr] (nullptr: the same as Rg) and the
// targets Rt[np][nr]; rows3: also the raw gradients (variant 3's rows).
__global__ void k_closure_rows(const double* Rg, const double* Rgf, const double* Rt, int np, size_t nr,
                               double delta2, float* X, size_t stride, int rows3) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nr; q += (size_t)gridDim.x * blockDim.x) {
        double A[9], G[9], f[8], S5[5], J3[3];
        if (Rgf) {
#pragma unroll
            for (int r = 0; r < 9; r++) {
                A[r] = Rgf[(size_t)r * nr + q];
                G[r] = Rgf[(size_t)(9 + r) * nr + q];
            }
            closure_features<double>(A, G, f, S5, J3);
#pragma unroll
            for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_SF + r) * stride + q] = (float)S5[r];
#pragma unroll
            for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_JF + r) * stride + q] = (float)J3[r];
        }
#pragma unroll
        for (int r = 0; r < 9; r++) {
            A[r] = Rg[(size_t)r * nr + q];
            G[r] = Rg[(size_t)(9 + r) * nr + q];
        }
        const double n = closure_features<double>(A, G, f, S5, J3);
        if (!Rgf) {
#pragma unroll
            for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_SF + r) * stride + q] = (float)S5[r];
#pragma unroll
            for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_JF + r) * stride + q] = (float)J3[r];
        }
#pragma unroll
        for (int r = 0; r < 8; r++) X[(size_t)(SPK_CLOSURE_ROW_FEAT + r) * stride + q] = (float)f[r];
#pragma unroll
        for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_S + r) * stride + q] = (float)S5[r];
#pragma unroll
        for (int r = 0; r < 3; r++) X[(size_t)(SPK_CLOSURE_ROW_J + r) * stride + q] = (float)J3[r];
        X[(size_t)SPK_CLOSURE_ROW_SCALE * stride + q] = (float)(delta2 * n);
#pragma unroll
        for (int r = 0; r < 5; r++) X[(size_t)(SPK_CLOSURE_ROW_TT + r) * stride + q] = (float)Rt[(size_t)r * nr + q];
#pragma unroll
        for (int r = 0; r < 3; r++)
            X[(size_t)(SPK_CLOSURE_ROW_TE + r) * stride + q] = np == 8 ? (float)Rt[(size_t)(5 + r) * nr + q] : 0.f;
        if (rows3) {
#pragma unroll
            for (int r = 0; r < 9; r++) {
                X[(size_t)(SPK_CLOSURE_ROW_A + r) * stride + q] = (float)A[r];
                X[(size_t)(SPK_CLOSURE_ROW_G + r) * stride + q] = (float)G[r];
            }
        }
    }
}

// Products of the x-forward pass (pass layout, kept modes) into the state
// layout in FP64, zero at masked modes.
template <typename T>
__global__ void k_products_out(const DevGrid g, const C2<T>* nl, int np, double2* P) {
    const size_t nc = g.nc;
    for (size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gi < nc * np; gi += (size_t)gridDim.x * blockDim.x) {
        const int ch = (int)(gi / nc);
        const size_t id = gi - (size_t)ch * nc;
        const int k = (int)(id % g.nzh);
        const size_t rr = id / g.nzh;
        const int j = (int)(rr % g.ny), i = (int)(rr / g.ny);
        double2 v = make_double2(0.0, 0.0);
        if (g.mx[i] * g.my[j] * g.mz[k] != 0.0) {
            const C2<T> x = nl[(size_t)ch * g.ncs + ((size_t)i * g.ny + j) * g.nzs + k];
            v = make_double2((double)x.x, (double)x.y);
        }
        P[gi] = v;
    }
}

}  // namespace spk

// ---------------------------------------------------------------------------
// variant 3, the tensor network (spk_closure3.cuh)
// ---------------------------------------------------------------------------
namespace spk {

// FP32 parameters -> the packed BF16 image (forward rows, biases, transposes)
__global__ void k_closure3_pack(const float* __restrict__ P, unsigned char* img) {
    uint16_t* w1 = (uint16_t*)(img + C3_OFF_W1);
    uint16_t* w2 = (uint16_t*)(img + C3_OFF_W2);
    uint16_t* w3 = (uint16_t*)(img + C3_OFF_W3);
    uint16_t* w4 = (uint16_t*)(img + C3_OFF_W4);
    float* b = (float*)(img + C3_OFF_B);
    uint16_t* w2t = (uint16_t*)(img + C3_OFF_W2T);
    uint16_t* w3t = (uint16_t*)(img + C3_OFF_W3T);
    uint16_t* w4t = (uint16_t*)(img + C3_OFF_W4T);
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int i = i0; i < 64 * C3_LD1; i += st) {
        const int r = i / C3_LD1, k = i % C3_LD1;
        w1[i] = k < C3_NI ? c3_bf(P[C3_W1 + r * C3_NI + k]) : (uint16_t)0;
    }
    for (int i = i0; i < 64 * C3_LDH; i += st) {
        const int r = i / C3_LDH, k = i % C3_LDH;
        w2[i] = k < 64 ? c3_bf(P[C3_W2 + r * 64 + k]) : (uint16_t)0;
        w3[i] = k < 64 ? c3_bf(P[C3_W3 + r * 64 + k]) : (uint16_t)0;
        // transposes: row = input i, column = output o
        w2t[i] = k < 64 ? c3_bf(P[C3_W2 + k * 64 + r]) : (uint16_t)0;
        w3t[i] = k < 64 ? c3_bf(P[C3_W3 + k * 64 + r]) : (uint16_t)0;
    }
    for (int i = i0; i < 16 * C3_LDH; i += st) {
        const int r = i / C3_LDH, k = i % C3_LDH;
        w4[i] = (r < C3_NO && k < 64) ? c3_bf(P[C3_W4 + r * 64 + k]) : (uint16_t)0;
    }
    for (int i = i0; i < 64 * C3_LD4T; i += st) {
        const int r = i / C3_LD4T, k = i % C3_LD4T;
        w4t[i] = k < C3_NO ? c3_bf(P[C3_W4 + k * 64 + r]) : (uint16_t)0;
    }
    for (int i = i0; i < 3 * 64 + 16; i += st) {
        float v;
        if (i < 64) v = P[C3_B1 + i];
        else if (i < 128) v = P[C3_B2 + i - 64];
        else if (i < 192) v = P[C3_B3 + i - 128];
        else v = i - 192 < C3_NO ? P[C3_B4 + i - 192] : 0.f;
        b[i] = v;
    }
}

#define C3_CH 64                 // samples per chunk: 16 per warp
#define C3_SLD 72                // staging row: 64 samples + 8 (conflict-free fragment loads)
// shared memory of the gradient kernel (bytes)
enum {
    C3G_IMG = 0,
    C3G_XT = C3G_IMG + C3_ALL_BYTES,               // xT [32][72] BF16 (rows >= 18 zero)
    C3G_H1 = C3G_XT + 32 * C3_SLD * 2,              // h1T h2T h3T d1T d2T d3T [64][72]
    C3G_D4 = C3G_H1 + 6 * 64 * C3_SLD * 2,          // d4T [16][72] (rows >= 12 zero)
    C3G_GW = C3G_D4 + 16 * C3_SLD * 2,              // gW1[64][32] gW2[64][64] gW3[64][64] gW4[16][64] FP32
    C3G_GB = C3G_GW + (64 * 32 + 2 * 64 * 64 + 16 * 64) * 4,   // gb [64 + 64 + 64 + 16]
    C3G_OS = C3G_GB + 208 * 4,                      // outputs [64][12]
    C3G_RED = C3G_OS + C3_CH * C3_NO * 4,           // loss reduction [128]
    C3G_BYTES = C3G_RED + 128 * 4
};

struct Train3Args {
    const float* X;          // sample rows (SPK_CLOSURE3_ROWS)
    size_t n, stride, m;
    int minibatch;
    unsigned long long a, c, base;
    const unsigned char* img;   // packed image of the current parameters
    float w0, w1, w2;
    float* partial;          // [gridDim.x][C3_NP + 1]
};

// BF16 pair (row f, f+1 of a [feature][sample] staging array at sample s)
__device__ __forceinline__ uint32_t c3_col2(const uint16_t* T, int f, int s) {
    return (uint32_t)T[f * C3_SLD + s] | ((uint32_t)T[(f + 1) * C3_SLD + s] << 16);
}
// the packed A chunks (rows s0+g, s0+g+8) into [feature][sample] staging
__device__ __forceinline__ void c3_stage(const uint32_t (&h)[4][4], uint16_t* T, int s0, int g, int t) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        const int f = 16 * kk + 2 * t;
        T[f * C3_SLD + s0 + g] = (uint16_t)h[kk][0];
        T[(f + 1) * C3_SLD + s0 + g] = (uint16_t)(h[kk][0] >> 16);
        T[f * C3_SLD + s0 + g + 8] = (uint16_t)h[kk][1];
        T[(f + 1) * C3_SLD + s0 + g + 8] = (uint16_t)(h[kk][1] >> 16);
        T[(f + 8) * C3_SLD + s0 + g] = (uint16_t)h[kk][2];
        T[(f + 9) * C3_SLD + s0 + g] = (uint16_t)(h[kk][2] >> 16);
        T[(f + 8) * C3_SLD + s0 + g + 8] = (uint16_t)h[kk][3];
        T[(f + 9) * C3_SLD + s0 + g + 8] = (uint16_t)(h[kk][3] >> 16);
    }
}
// back-propagated errors: acc x (1 - h^2) with h the staged BF16 activation,
// rounded to BF16 as the next A chunks and staged for the weight gradients
__device__ __forceinline__ void c3_bwd_act(const float (&acc)[8][4], const uint16_t* H, uint16_t* D, uint32_t (&d)[4][4],
                                           int s0, int g, int t) {
    auto hv = [&](int f, int s) { return __uint_as_float((uint32_t)H[f * C3_SLD + s] << 16); };
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int f = 8 * j + 2 * t;
        float v[4];
        v[0] = acc[j][0] * (1.f - hv(f, s0 + g) * hv(f, s0 + g));
        v[1] = acc[j][1] * (1.f - hv(f + 1, s0 + g) * hv(f + 1, s0 + g));
        v[2] = acc[j][2] * (1.f - hv(f, s0 + g + 8) * hv(f, s0 + g + 8));
        v[3] = acc[j][3] * (1.f - hv(f + 1, s0 + g + 8) * hv(f + 1, s0 + g + 8));
        const uint32_t p0 = c3_pack(v[0], v[1]), p1 = c3_pack(v[2], v[3]);
        d[j >> 1][(j & 1) * 2] = p0;
        d[j >> 1][(j & 1) * 2 + 1] = p1;
        D[f * C3_SLD + s0 + g] = (uint16_t)p0;
        D[(f + 1) * C3_SLD + s0 + g] = (uint16_t)(p0 >> 16);
        D[f * C3_SLD + s0 + g + 8] = (uint16_t)p1;
        D[(f + 1) * C3_SLD + s0 + g + 8] = (uint16_t)(p1 >> 16);
    }
}

// Loss and gradient partials of one CTA: chunks of 64 samples, forward and
// backward per warp on the tensor cores, then the chunk's weight gradients
// dW = sum_s delta_s (x) h_s as MMAs over the staged [feature][sample]
// arrays (M = outputs, N = inputs, K = samples), accumulated in shared FP32
// by fixed warps in a fixed order: deterministic.
__global__ void __launch_bounds__(128, 1) k_closure3_grad(const __grid_constant__ Train3Args a) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint16_t* xT = (uint16_t*)(sm + C3G_XT);
    uint16_t* h1T = (uint16_t*)(sm + C3G_H1);
    uint16_t* h2T = h1T + 64 * C3_SLD;
    uint16_t* h3T = h2T + 64 * C3_SLD;
    uint16_t* d1T = h3T + 64 * C3_SLD;
    uint16_t* d2T = d1T + 64 * C3_SLD;
    uint16_t* d3T = d2T + 64 * C3_SLD;
    uint16_t* d4T = (uint16_t*)(sm + C3G_D4);
    float* gW1 = (float*)(sm + C3G_GW);
    float* gW2 = gW1 + 64 * 32;
    float* gW3 = gW2 + 64 * 64;
    float* gW4 = gW3 + 64 * 64;
    float* gb = (float*)(sm + C3G_GB);
    float* Os = (float*)(sm + C3G_OS);
    float* red = (float*)(sm + C3G_RED);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    {
        const uint4* src = (const uint4*)a.img;
        uint4* dst = (uint4*)sm;
        for (int i = tid; i < C3_ALL_BYTES / 16; i += 128) dst[i] = src[i];
        uint32_t* z = (uint32_t*)(sm + C3G_XT);   // staging and accumulators start at zero
        for (int i = tid; i < (C3G_RED - C3G_XT) / 4; i += 128) z[i] = 0u;
    }
    __syncthreads();
    const C3Img m(sm);
    const uint16_t* w2t = (const uint16_t*)(sm + C3_OFF_W2T);
    const uint16_t* w3t = (const uint16_t*)(sm + C3_OFF_W3T);
    const uint16_t* w4t = (const uint16_t*)(sm + C3_OFF_W4T);
    const int s0 = 16 * warp;
    float lsum = 0.f;
    const size_t nch = (a.m + C3_CH - 1) / C3_CH;
    for (size_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        // inputs: lane l < 16 takes sample s0 + l
        float nrm = 1.f, sc = 0.f;
        size_t sidx = 0;
        bool valid = false;
        if (lane < 16) {
            const size_t r = ch * C3_CH + s0 + lane;
            valid = r < a.m;
            if (valid) sidx = a.minibatch ? (size_t)((a.a * ((a.base + r) % a.n) + a.c) % a.n) : r;
            float A[18], f[8], S5[5], J3[3];
#pragma unroll
            for (int i = 0; i < 18; i++) A[i] = valid ? a.X[(size_t)(SPK_CLOSURE_ROW_A + i) * a.stride + sidx] : 0.f;
            nrm = closure_features<float>(A, A + 9, f, S5, J3);
#pragma unroll
            for (int i = 0; i < 18; i++) xT[i * C3_SLD + s0 + lane] = c3_bf(A[i] / nrm);
            sc = valid ? a.X[(size_t)SPK_CLOSURE_ROW_SCALE * a.stride + sidx] * nrm : 0.f;
        }
        __syncwarp();
        uint32_t ax[2][4];
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            ax[kk][0] = c3_col2(xT, 16 * kk + 2 * t, s0 + g);
            ax[kk][1] = c3_col2(xT, 16 * kk + 2 * t, s0 + g + 8);
            ax[kk][2] = c3_col2(xT, 16 * kk + 2 * t + 8, s0 + g);
            ax[kk][3] = c3_col2(xT, 16 * kk + 2 * t + 8, s0 + g + 8);
        }
        // forward, staging the rounded activations
        float acc[8][4], o[2][4];
        uint32_t h[4][4], q[4][4];
        c3_layer<2, 8, C3_LD1>(m.w1, m.b1, ax, acc, g, t);
        c3_act(acc, h);
        c3_stage(h, h1T, s0, g, t);
        c3_layer<4, 8, C3_LDH>(m.w2, m.b2, h, acc, g, t);
        c3_act(acc, q);
        c3_stage(q, h2T, s0, g, t);
        c3_layer<4, 8, C3_LDH>(m.w3, m.b3, q, acc, g, t);
        c3_act(acc, h);
        c3_stage(h, h3T, s0, g, t);
        c3_layer<4, 2, C3_LDH>(m.w4, m.b4, h, o, g, t);
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int col = 8 * j + 2 * t;
            if (col < C3_NO) {
                Os[(s0 + g) * C3_NO + col] = o[j][0];
                Os[(s0 + g) * C3_NO + col + 1] = o[j][1];
                Os[(s0 + g + 8) * C3_NO + col] = o[j][2];
                Os[(s0 + g + 8) * C3_NO + col + 1] = o[j][3];
            }
        }
        __syncwarp();
        // loss and d loss / d o per sample (include/spooky_b200.h)
        if (lane < 16) {
            float tT[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, tE[3] = {0.f, 0.f, 0.f};
            float Sf[5] = {0.f, 0.f, 0.f, 0.f, 0.f}, Jf[3] = {0.f, 0.f, 0.f};
            if (valid) {
#pragma unroll
                for (int r = 0; r < 5; r++) {
                    tT[r] = a.X[(size_t)(SPK_CLOSURE_ROW_TT + r) * a.stride + sidx];
                    Sf[r] = a.X[(size_t)(SPK_CLOSURE_ROW_SF + r) * a.stride + sidx];
                }
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    tE[r] = a.X[(size_t)(SPK_CLOSURE_ROW_TE + r) * a.stride + sidx];
                    Jf[r] = a.X[(size_t)(SPK_CLOSURE_ROW_JF + r) * a.stride + sidx];
                }
            }
            float s[C3_NO];
#pragma unroll
            for (int i = 0; i < C3_NO; i++) s[i] = sc * Os[(s0 + lane) * C3_NO + i];
            const float tr = (s[0] + s[3] + s[5]) * (1.f / 3.f);
            float e[5] = {s[0] - tr - tT[0], s[1] - tT[1], s[2] - tT[2], s[3] - tr - tT[3], s[4] - tT[4]};
            float eE[3] = {0.5f * (s[9] - s[11]) - tE[0], 0.5f * (s[10] - s[7]) - tE[1], 0.5f * (s[6] - s[8]) - tE[2]};
            const float ezz = -(e[0] + e[3]), Sfzz = -(Sf[0] + Sf[3]);
            const float fro = e[0] * e[0] + e[3] * e[3] + ezz * ezz + 2.f * (e[1] * e[1] + e[2] * e[2] + e[4] * e[4]);
            const float emf = eE[0] * eE[0] + eE[1] * eE[1] + eE[2] * eE[2];
            const float eJ = eE[0] * Jf[0] + eE[1] * Jf[1] + eE[2] * Jf[2];
            const float dP = -(e[0] * Sf[0] + e[3] * Sf[3] + ezz * Sfzz + 2.f * (e[1] * Sf[1] + e[2] * Sf[2] + e[4] * Sf[4])) - eJ;
            if (valid) lsum += a.w0 * fro + a.w1 * emf + a.w2 * dP * dP;
            const float p2 = a.w2 * 2.f * dP;
            float g5[5], gE[3], gs[C3_NO];
            g5[0] = a.w0 * (2.f * e[0] - 2.f * ezz) - p2 * (Sf[0] - Sfzz);
            g5[3] = a.w0 * (2.f * e[3] - 2.f * ezz) - p2 * (Sf[3] - Sfzz);
            g5[1] = a.w0 * 4.f * e[1] - p2 * 2.f * Sf[1];
            g5[2] = a.w0 * 4.f * e[2] - p2 * 2.f * Sf[2];
            g5[4] = a.w0 * 4.f * e[4] - p2 * 2.f * Sf[4];
#pragma unroll
            for (int r = 0; r < 3; r++) gE[r] = a.w1 * 2.f * eE[r] - p2 * Jf[r];
            gs[0] = (2.f * g5[0] - g5[3]) * (1.f / 3.f);
            gs[3] = (2.f * g5[3] - g5[0]) * (1.f / 3.f);
            gs[5] = -(g5[0] + g5[3]) * (1.f / 3.f);
            gs[1] = g5[1]; gs[2] = g5[2]; gs[4] = g5[4];
            gs[9] = 0.5f * gE[0]; gs[11] = -0.5f * gE[0];
            gs[10] = 0.5f * gE[1]; gs[7] = -0.5f * gE[1];
            gs[6] = 0.5f * gE[2]; gs[8] = -0.5f * gE[2];
#pragma unroll
            for (int i = 0; i < C3_NO; i++) d4T[i * C3_SLD + s0 + lane] = c3_bf(valid ? sc * gs[i] : 0.f);
        }
        __syncwarp();
        // backward: delta3 = (delta4 W4) (1 - h3^2), delta2, delta1 likewise
        {
            uint32_t d4[1][4];
            d4[0][0] = c3_col2(d4T, 2 * t, s0 + g);
            d4[0][1] = c3_col2(d4T, 2 * t, s0 + g + 8);
            d4[0][2] = c3_col2(d4T, 2 * t + 8, s0 + g);
            d4[0][3] = c3_col2(d4T, 2 * t + 8, s0 + g + 8);
            c3_layer<1, 8, C3_LD4T>(w4t, nullptr, d4, acc, g, t);
        }
        c3_bwd_act(acc, h3T, d3T, h, s0, g, t);
        c3_layer<4, 8, C3_LDH>(w3t, nullptr, h, acc, g, t);
        c3_bwd_act(acc, h2T, d2T, q, s0, g, t);
        c3_layer<4, 8, C3_LDH>(w2t, nullptr, q, acc, g, t);
        c3_bwd_act(acc, h1T, d1T, h, s0, g, t);
        __syncthreads();
        // weight gradients of the chunk: 16 + 32 + 32 + 8 tiles of 16 x 8,
        // tile i by warp i % 4
#pragma unroll 1
        for (int tile = warp; tile < 88; tile += 4) {
            const uint16_t *D, *H;
            float* G;
            int mt, nt, ldg;
            if (tile < 16) { D = d1T; H = xT; G = gW1; ldg = 32; mt = tile >> 2; nt = tile & 3; }
            else if (tile < 48) { D = d2T; H = h1T; G = gW2; ldg = 64; mt = (tile - 16) >> 3; nt = (tile - 16) & 7; }
            else if (tile < 80) { D = d3T; H = h2T; G = gW3; ldg = 64; mt = (tile - 48) >> 3; nt = (tile - 48) & 7; }
            else { D = d4T; H = h3T; G = gW4; ldg = 64; mt = 0; nt = tile - 80; }
            float* g0 = G + (16 * mt + g) * ldg + 8 * nt + 2 * t;
            float* g1 = g0 + 8 * ldg;
            float c[4] = {g0[0], g0[1], g1[0], g1[1]};
            const uint16_t* dr0 = D + (16 * mt + g) * C3_SLD + 2 * t;
            const uint16_t* dr1 = dr0 + 8 * C3_SLD;
            const uint16_t* hr = H + (8 * nt + g) * C3_SLD + 2 * t;
#pragma unroll
            for (int ks = 0; ks < C3_CH / 16; ks++) {
                uint32_t af[4];
                af[0] = *reinterpret_cast<const uint32_t*>(dr0 + 16 * ks);
                af[1] = *reinterpret_cast<const uint32_t*>(dr1 + 16 * ks);
                af[2] = *reinterpret_cast<const uint32_t*>(dr0 + 16 * ks + 8);
                af[3] = *reinterpret_cast<const uint32_t*>(dr1 + 16 * ks + 8);
                c3_mma(c, af, *reinterpret_cast<const uint32_t*>(hr + 16 * ks),
                       *reinterpret_cast<const uint32_t*>(hr + 16 * ks + 8));
            }
            g0[0] = c[0]; g0[1] = c[1]; g1[0] = c[2]; g1[1] = c[3];
        }
        // bias gradients: sums of the staged errors over the chunk
        for (int p = tid; p < 208; p += 128) {
            const uint16_t* D = p < 64 ? d1T + p * C3_SLD
                              : (p < 128 ? d2T + (p - 64) * C3_SLD : (p < 192 ? d3T + (p - 128) * C3_SLD : d4T + (p - 192) * C3_SLD));
            float sacc = 0.f;
            for (int s = 0; s < C3_CH; s++) sacc += __uint_as_float((uint32_t)D[s] << 16);
            gb[p] += sacc;
        }
        __syncthreads();   // the next chunk overwrites the staging
    }
    float* out = a.partial + (size_t)blockIdx.x * (C3_NP + 1);
    for (int p = tid; p < C3_NP; p += 128) {
        float v;
        if (p < C3_B1) v = gW1[(p / C3_NI) * 32 + p % C3_NI];
        else if (p < C3_W2) v = gb[p - C3_B1];
        else if (p < C3_B2) v = gW2[p - C3_W2];
        else if (p < C3_W3) v = gb[64 + p - C3_B2];
        else if (p < C3_B3) v = gW3[p - C3_W3];
        else if (p < C3_W4) v = gb[128 + p - C3_B3];
        else if (p < C3_B4) v = gW4[p - C3_W4];
        else v = gb[192 + p - C3_B4];
        out[p] = v;
    }
    red[tid] = lsum;
    __syncthreads();
    if (tid == 0) {
        float s = 0.f;
        for (int i = 0; i < 128; i++) s += red[i];
        out[C3_NP] = s;
    }
}

// grad[p] = sum over CTAs of partial[b][p] / m (FP64, fixed order) for np
// parameters; the loss (entry np) to loss_out
__global__ void k_closure_reduce_n(const float* partial, int nblk, int np, double inv_m, float* grad, float* loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > np) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += (double)partial[(size_t)b * (np + 1) + p];
    if (p < np) grad[p] = (float)(s * inv_m);
    else if (loss_out) *loss_out = (float)(s * inv_m);
}

// One Adam step over np parameters (as k_closure_adam)
__global__ void k_closure_adam_n(float* params, const float* grad, float* m, float* v, int np, int t, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const double b1 = 0.9, b2 = 0.999;
    const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
    const float g = grad[p];
    const float mm = (float)(b1 * m[p] + (1.0 - b1) * g);
    const float vv = (float)(b2 * v[p] + (1.0 - b2) * (double)g * g);
    m[p] = mm;
    v[p] = vv;
    params[p] -= (float)(lr * (mm / c1) / (sqrt(vv / c2) + 1e-8));
}

}  // namespace spk
