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
// targets Rt[np][nr].
__global__ void k_closure_rows(const double* Rg, const double* Rgf, const double* Rt, int np, size_t nr,
                               double delta2, float* X, size_t stride) {
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
