// spk_closure3.cuh -- variant 3 of the learned closure, the tensor network
// (definition in include/spooky_b200.h, SPK_CLOSURE3_*): 18 dimensionless
// gradients -> 64 -> 64 -> 64 -> 12 with tanh, BF16 operands and FP32
// accumulation on the tensor cores (mma.sync m16n8k16).
//
// One warp evaluates 16 points (the M = 16 rows of an MMA tile).  The
// accumulator fragment of a layer (rows g, g+8; columns 2t, 2t+1 of each
// 8-column tile, g = lane/4, t = lane%4) is, pair by pair, the A fragment of
// the next layer's 16-column K chunk, so activations never leave the
// registers: bias + tanh + BF16 packing turn one layer's output into the
// next layer's input.  Weights sit in shared memory as BF16 rows padded to
// 40 / 72 / 24 elements, which makes every B-fragment load (row 8j+g, word
// t) hit 32 distinct banks.
//
// Used by the z pass (fused inference, GEN 3) and by the trainer
// (forward, backward and weight gradients, all on the tensor cores).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace spk {

enum { C3_NI = 18, C3_NH = 64, C3_NO = 12 };
// parameter offsets: W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[12][64] b4[12]
enum {
    C3_W1 = 0,
    C3_B1 = C3_W1 + C3_NH * C3_NI,
    C3_W2 = C3_B1 + C3_NH,
    C3_B2 = C3_W2 + C3_NH * C3_NH,
    C3_W3 = C3_B2 + C3_NH,
    C3_B3 = C3_W3 + C3_NH * C3_NH,
    C3_W4 = C3_B3 + C3_NH,
    C3_B4 = C3_W4 + C3_NO * C3_NH,
    C3_NP = C3_B4 + C3_NO
};
// packed image of the network (bytes, each part 16-byte aligned):
// forward rows W1p[64][40] (k < 18 set), W2p, W3p [64][72], W4p[16][72]
// (rows < 12 set), biases b1 b2 b3 [64] and b4[16] in FP32; the trainer's
// transposes W2T, W3T [64][72] and W4T[64][24] follow.
enum {
    C3_LD1 = 40,
    C3_LDH = 72,
    C3_LD4T = 24,
    C3_OFF_W1 = 0,
    C3_OFF_W2 = C3_OFF_W1 + 64 * C3_LD1 * 2,
    C3_OFF_W3 = C3_OFF_W2 + 64 * C3_LDH * 2,
    C3_OFF_W4 = C3_OFF_W3 + 64 * C3_LDH * 2,
    C3_OFF_B = C3_OFF_W4 + 16 * C3_LDH * 2,
    C3_FWD_BYTES = C3_OFF_B + (3 * 64 + 16) * 4,
    C3_OFF_W2T = C3_FWD_BYTES,
    C3_OFF_W3T = C3_OFF_W2T + 64 * C3_LDH * 2,
    C3_OFF_W4T = C3_OFF_W3T + 64 * C3_LDH * 2,
    C3_ALL_BYTES = C3_OFF_W4T + 64 * C3_LD4T * 2
};
// z pass: the packed forward image, then one 80-byte row per point of a
// 128-point chunk (the inputs as 40 BF16, later the 12 FP32 outputs)
enum { C3_ZROW = 80, C3_ZCHUNK = 128, C3_ZBYTES = C3_FWD_BYTES + C3_ZCHUNK * C3_ZROW };
static_assert(C3_FWD_BYTES % 16 == 0 && C3_ALL_BYTES % 16 == 0 && C3_ZBYTES % 16 == 0, "image alignment");

__device__ __forceinline__ uint16_t c3_bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ uint32_t c3_pack(float lo, float hi) {
    return (uint32_t)c3_bf(lo) | ((uint32_t)c3_bf(hi) << 16);
}
__device__ __forceinline__ float c3_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float c3_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }
// full-accuracy FP32 tanh: its result is rounded to BF16 next, and an
// approximate tanh would move that rounding for a good share of activations
__device__ __forceinline__ float c3_tanh(float x) { return tanhf(x); }

// D += A B: A 16x16 (row), B 16x8 (col), BF16 operands, FP32 accumulators
__device__ __forceinline__ void c3_mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc[j] = bias + A W^T over NT output tiles of 8 and KC input chunks of 16;
// W row o at W + o*LD (BF16, k contiguous); bias nullptr: zero.
template <int KC, int NT, int LD>
__device__ __forceinline__ void c3_layer(const uint16_t* __restrict__ W, const float* __restrict__ bias,
                                         const uint32_t (&a)[KC][4], float (&acc)[NT][4], int g, int t) {
#pragma unroll
    for (int j = 0; j < NT; j++) {
        const float b0 = bias ? bias[8 * j + 2 * t] : 0.f, b1 = bias ? bias[8 * j + 2 * t + 1] : 0.f;
        acc[j][0] = b0; acc[j][1] = b1; acc[j][2] = b0; acc[j][3] = b1;
        const uint16_t* wr = W + (8 * j + g) * LD + 2 * t;
#pragma unroll
        for (int kk = 0; kk < KC; kk++) {
            const uint32_t w0 = *reinterpret_cast<const uint32_t*>(wr + 16 * kk);
            const uint32_t w1 = *reinterpret_cast<const uint32_t*>(wr + 16 * kk + 8);
            c3_mma(acc[j], a[kk], w0, w1);
        }
    }
}

// tanh of 8 output tiles, packed to BF16 as the next layer's 4 A chunks
__device__ __forceinline__ void c3_act(const float (&acc)[8][4], uint32_t (&a)[4][4]) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        a[kk][0] = c3_pack(c3_tanh(acc[2 * kk][0]), c3_tanh(acc[2 * kk][1]));
        a[kk][1] = c3_pack(c3_tanh(acc[2 * kk][2]), c3_tanh(acc[2 * kk][3]));
        a[kk][2] = c3_pack(c3_tanh(acc[2 * kk + 1][0]), c3_tanh(acc[2 * kk + 1][1]));
        a[kk][3] = c3_pack(c3_tanh(acc[2 * kk + 1][2]), c3_tanh(acc[2 * kk + 1][3]));
    }
}

struct C3Img {
    const uint16_t *w1, *w2, *w3, *w4;
    const float *b1, *b2, *b3, *b4;
    __device__ __forceinline__ explicit C3Img(const unsigned char* p)
        : w1((const uint16_t*)(p + C3_OFF_W1)), w2((const uint16_t*)(p + C3_OFF_W2)),
          w3((const uint16_t*)(p + C3_OFF_W3)), w4((const uint16_t*)(p + C3_OFF_W4)),
          b1((const float*)(p + C3_OFF_B)), b2(b1 + 64), b3(b1 + 128), b4(b1 + 192) {}
};

// The whole network on one warp's 16 rows: input fragments ax (2 K chunks)
// to the output tiles o (columns 0..15, 12 used).
__device__ __forceinline__ void c3_forward(const C3Img& m, const uint32_t (&ax)[2][4], float (&o)[2][4], int g, int t) {
    float acc[8][4];
    uint32_t h[4][4], h2[4][4];
    c3_layer<2, 8, C3_LD1>(m.w1, m.b1, ax, acc, g, t);
    c3_act(acc, h);
    c3_layer<4, 8, C3_LDH>(m.w2, m.b2, h, acc, g, t);
    c3_act(acc, h2);
    c3_layer<4, 8, C3_LDH>(m.w3, m.b3, h2, acc, g, t);
    c3_act(acc, h);
    c3_layer<4, 2, C3_LDH>(m.w4, m.b4, h, o, g, t);
}

// Model terms of one point from its outputs o[12] (include/spooky_b200.h):
// tau[5] and e[3] after the backscatter ramp; nu, eta: the dt rule's rates.
__device__ __forceinline__ void c3_terms(const float* o, float delta2, float n, float Szz, const float* S5,
                                         const float* J3, bool mhd, float* tau, float* e, float* nu, float* eta) {
    const float sc = delta2 * n * n;
    float s[C3_NO];
#pragma unroll
    for (int i = 0; i < C3_NO; i++) s[i] = sc * o[i];
    const float tr = (s[0] + s[3] + s[5]) * (1.f / 3.f);
    const float dT[5] = {s[0] - tr, s[1], s[2], s[3] - tr, s[4]};
    float dE[3] = {0.5f * (s[9] - s[11]), 0.5f * (s[10] - s[7]), 0.5f * (s[6] - s[8])};
    if (!mhd) dE[0] = dE[1] = dE[2] = 0.f;
    const float dTzz = -(dT[0] + dT[3]);
    const float TS = dT[0] * S5[0] + dT[3] * S5[3] + dTzz * Szz + 2.f * (dT[1] * S5[1] + dT[2] * S5[2] + dT[4] * S5[4]);
    const float T2 = dT[0] * dT[0] + dT[3] * dT[3] + dTzz * dTzz + 2.f * (dT[1] * dT[1] + dT[2] * dT[2] + dT[4] * dT[4]);
    const float S2 = S5[0] * S5[0] + S5[3] * S5[3] + Szz * Szz + 2.f * (S5[1] * S5[1] + S5[2] * S5[2] + S5[4] * S5[4]);
    const float EJ = dE[0] * J3[0] + dE[1] * J3[1] + dE[2] * J3[2];
    const float E2 = dE[0] * dE[0] + dE[1] * dE[1] + dE[2] * dE[2];
    const float J2 = J3[0] * J3[0] + J3[1] * J3[1] + J3[2] * J3[2];
    const float P = -TS - EJ, Pm = sqrtf(T2) * sqrtf(S2) + sqrtf(E2) * sqrtf(J2);
    const float r = fminf(fmaxf(P / (0.1f * Pm + 1e-30f), 0.f), 1.f);
#pragma unroll
    for (int k = 0; k < 5; k++) tau[k] = r * dT[k];
#pragma unroll
    for (int k = 0; k < 3; k++) e[k] = r * dE[k];
    *nu = r * sqrtf(T2) / (2.f * n);
    *eta = mhd ? r * sqrtf(E2) / n : 0.f;
}

// z pass, one 128-point chunk, phase 1: thread p writes point p's inputs x =
// (A, G)/n as a BF16 row (cols 18..31 zero; the row's last 8 are padding).
__device__ __forceinline__ void c3_put_inputs(unsigned char* rows, int p, const float* A, const float* G) {
    float f[8], S5[5], J3[3];
    const float n = closure_features<float>(A, G, f, S5, J3);
    uint32_t* w = reinterpret_cast<uint32_t*>(rows + (size_t)p * C3_ZROW);
#pragma unroll
    for (int q = 0; q < 4; q++) w[q] = c3_pack(A[2 * q] / n, A[2 * q + 1] / n);
    w[4] = c3_pack(A[8] / n, G[0] / n);
#pragma unroll
    for (int q = 0; q < 4; q++) w[5 + q] = c3_pack(G[2 * q + 1] / n, G[2 * q + 2] / n);
#pragma unroll
    for (int q = 9; q < 16; q++) w[q] = 0u;
}

// phase 2: warp w runs the network on rows [32w, 32w + 32) and leaves the
// 12 FP32 outputs of each row at the row's start.
__device__ __forceinline__ void c3_chunk_mlp(const unsigned char* img, unsigned char* rows, int warp, int lane) {
    const C3Img m(img);
    const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int tt = 0; tt < 2; tt++) {
        const int p0 = 32 * warp + 16 * tt;
        uint32_t ax[2][4];
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            const unsigned char* r0 = rows + (size_t)(p0 + g) * C3_ZROW + (16 * kk + 2 * t) * 2;
            const unsigned char* r1 = r0 + 8 * C3_ZROW;
            ax[kk][0] = *reinterpret_cast<const uint32_t*>(r0);
            ax[kk][1] = *reinterpret_cast<const uint32_t*>(r1);
            ax[kk][2] = *reinterpret_cast<const uint32_t*>(r0 + 16);
            ax[kk][3] = *reinterpret_cast<const uint32_t*>(r1 + 16);
        }
        float o[2][4];
        c3_forward(m, ax, o, g, t);
        __syncwarp();   // every lane has read its inputs before the rows are overwritten
        float* o0 = reinterpret_cast<float*>(rows + (size_t)(p0 + g) * C3_ZROW);
        float* o1 = reinterpret_cast<float*>(rows + (size_t)(p0 + g + 8) * C3_ZROW);
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int col = 8 * j + 2 * t;
            if (col < C3_NO) {
                o0[col] = o[j][0]; o0[col + 1] = o[j][1];
                o1[col] = o[j][2]; o1[col + 1] = o[j][3];
            }
        }
    }
}

}  // namespace spk
