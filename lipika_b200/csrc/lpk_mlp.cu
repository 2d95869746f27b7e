// lpk_mlp.cu — the learned warm start of the emission-time solve, and the
// converged solver it serves.
//
// The reference solves the emission time with two fixed-point iterations
// from t - 70 ms (src/channel/mod.rs:49-101). Where a converged solve is
// wanted (the delay truth, or a solver that iterates to a residual), each
// sample starts from one of:
//   LAG        the reference's initial guess, t - 70 ms;
//   GEOMETRIC  the range at the reception time, R(t) / c (trajectory table);
//   LEARNED    the scene's surrogate: a function of the transmitter's
//              circular-orbit elements, the receiver's ECEF position and the
//              reception time t alone. An analytic layer turns (elements,
//              receiver, t) into 16 features — the raw inputs plus the
//              orbit's line of sight, range and range rate at t — and a
//              16 -> 64 -> 64 -> 64 -> 1 tanh MLP predicts the light-time
//              correction τ - R_orbit(t)/c; the start is R_orbit(t)/c plus
//              that correction. One network serves every (transmitter,
//              receiver) pair of a scene.
// Fixed-point or Newton iterations then finish the solve to the requested
// tolerance; a start that does not converge within the budget falls back to
// the LAG start, and the distance of every start from the converged delay
// is reported (the surrogate is judged, never trusted).
//
// The network is trained on this GPU from delays the converged solver
// itself produces. Inference runs on the 5th-generation tensor cores
// (tcgen05.mma, BF16 operands, FP32 accumulator in TMEM, 128-row tiles).
// Training is latency-bound (a batch is a few thousand rows), so its
// forward, backward and weight-gradient products are BF16 mma.sync tiles
// held in each warp's registers and the block's shared memory; Adam updates
// FP32 master weights. Rounding points (BF16: the inputs, W1-W3, the first
// two hidden layers and the three pre-activation gradients as MMA operands;
// everything else FP32) are restated in oracle/mlp_ref.py.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "lpk_internal.h"
#include "lpk_split.cuh"

namespace lpk {
namespace {

constexpr int kF = 16;   // features
constexpr int kH = 64;   // hidden width (three hidden layers)
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kH, kOffW4 = kOffB3 + kH, kOffB4 = kOffW4 + kH;
constexpr int kParams = kOffB4 + 1;  // 9473
constexpr int kNorm = 2 * kF + 2;    // feature means, feature stds, target mean, target std (µs)
static_assert(kParams == LPK_MLP_N_PARAMS && kF == LPK_MLP_N_FEATURES && kNorm == LPK_MLP_N_NORM, "ABI sizes");
constexpr int kLdW1 = kF + 8;        // padded row strides (bf16 elements) of the shared weight tiles
constexpr int kLdW = kH + 8;
constexpr int kRowsPerBlock = 128;   // 8 warps x 16 rows per block step (training)
constexpr int kLdR = kRowsPerBlock + 8;

struct __align__(16) MlpWeights {
    __nv_bfloat16 w1[kH][kLdW1];  // W1 (out x in)
    __nv_bfloat16 w2[kH][kLdW];   // W2 (out x in) and transposed
    __nv_bfloat16 w2t[kH][kLdW];
    __nv_bfloat16 w3[kH][kLdW];   // W3 (out x in) and transposed
    __nv_bfloat16 w3t[kH][kLdW];
    float b1[kH], b2[kH], b3[kH], w4[kH], b4;
};

// One block step's weight-gradient operands, transposed so that the step's
// 128 rows are the contraction index: dW3 = dZ3^T H2, dW2 = dZ2^T H1,
// dW1 = dZ1^T X (each row of these arrays is one output or input column).
struct __align__(16) MlpStage {
    __nv_bfloat16 dz3t[kH][kLdR], h2t[kH][kLdR], dz2t[kH][kLdR], h1t[kH][kLdR], dz1t[kH][kLdR];
    __nv_bfloat16 xt[kF][kLdR];
    float db1[kH], db2[kH], db3[kH], dw4[kH], db4, loss;
};
constexpr size_t kWeightsBytes = (sizeof(MlpWeights) + 15) / 16 * 16;
constexpr size_t kGradSmem = kWeightsBytes + sizeof(MlpStage);

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld2(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// D = A(16x16, row) x B(16x8, col) + D, BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// FP32 master parameters -> shared weights (BF16 where the mma reads them).
__device__ void stage_weights(const float *__restrict__ p, MlpWeights &S) {
    for (int i = threadIdx.x; i < kH * kLdW1; i += blockDim.x) {
        const int o = i / kLdW1, k = i % kLdW1;
        S.w1[o][k] = __float2bfloat16_rn(k < kF ? p[kOffW1 + o * kF + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int o = i / kH, k = i % kH;
        const __nv_bfloat16 w2 = __float2bfloat16_rn(p[kOffW2 + i]), w3 = __float2bfloat16_rn(p[kOffW3 + i]);
        S.w2[o][k] = w2;
        S.w2t[k][o] = w2;
        S.w3[o][k] = w3;
        S.w3t[k][o] = w3;
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        S.b1[i] = p[kOffB1 + i];
        S.b2[i] = p[kOffB2 + i];
        S.b3[i] = p[kOffB3 + i];
        S.w4[i] = p[kOffW4 + i];
    }
    if (threadIdx.x == 0) S.b4 = p[kOffB4];
}

// A fragments (m16n8k16, rows g and g+8 of the warp's 16) of a 16 x 64
// activation held in accumulator layout: h[j][e] is column 8j + 2·tig + (e & 1)
// of row g (e < 2) or g + 8 (e >= 2).
__device__ __forceinline__ void act_fragments(const float h[8][4], uint32_t a[4][4]) {
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        a[kk][0] = pack2(h[2 * kk][0], h[2 * kk][1]);
        a[kk][1] = pack2(h[2 * kk][2], h[2 * kk][3]);
        a[kk][2] = pack2(h[2 * kk + 1][0], h[2 * kk + 1][1]);
        a[kk][3] = pack2(h[2 * kk + 1][2], h[2 * kk + 1][3]);
    }
}

// out = act(A W^T + bias) over the warp's 16 rows, 64 columns; W is 64 x 64
// (out x in) in shared memory with row stride kLdW.
__device__ __forceinline__ void layer64(const uint32_t a[4][4], const __nv_bfloat16 (*w)[kLdW], const float *bias,
                                        float out[8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {bias[8 * j + 2 * tig], bias[8 * j + 2 * tig + 1], bias[8 * j + 2 * tig],
                        bias[8 * j + 2 * tig + 1]};
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma16816(acc, a[kk], ld2(&w[8 * j + g][16 * kk + 2 * tig]), ld2(&w[8 * j + g][16 * kk + 8 + 2 * tig]));
#pragma unroll
        for (int e = 0; e < 4; ++e) out[j][e] = tanhf(acc[e]);
    }
}

// Forward pass of one warp's 16 rows. ax: the BF16 input fragments (rows g
// and g+8, features 2·tig, 2·tig+1, 2·tig+8, 2·tig+9). Leaves the three
// hidden layers' tanh outputs in accumulator layout and y for rows g (y[0])
// and g+8 (y[1]) in every thread of the group.
struct WarpAct {
    float h1[8][4], h2[8][4], h3[8][4];
};

__device__ __forceinline__ void warp_forward(const MlpWeights &S, const uint32_t ax[4], WarpAct &A, float y[2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {S.b1[8 * j + 2 * tig], S.b1[8 * j + 2 * tig + 1], S.b1[8 * j + 2 * tig],
                        S.b1[8 * j + 2 * tig + 1]};
        mma16816(acc, ax, ld2(&S.w1[8 * j + g][2 * tig]), ld2(&S.w1[8 * j + g][8 + 2 * tig]));
#pragma unroll
        for (int e = 0; e < 4; ++e) A.h1[j][e] = tanhf(acc[e]);
    }
    uint32_t a[4][4];
    act_fragments(A.h1, a);
    layer64(a, S.w2, S.b2, A.h2);
    act_fragments(A.h2, a);
    layer64(a, S.w3, S.b3, A.h3);
    float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float wa = S.w4[8 * j + 2 * tig], wb = S.w4[8 * j + 2 * tig + 1];
        s0 = fmaf(A.h3[j][0], wa, fmaf(A.h3[j][1], wb, s0));
        s1 = fmaf(A.h3[j][2], wa, fmaf(A.h3[j][3], wb, s1));
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    y[0] = s0 + S.b4;
    y[1] = s1 + S.b4;
}

// Sum of v over the 16 rows a warp holds (rows g and g+8 of every group):
// this thread's two elements, then across the eight groups.
__device__ __forceinline__ float rows_sum(float a, float b) {
    float v = a + b;
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// dZ = (dH = dZ_next W) ⊙ (1 - h²) over the warp's 16 rows; wt is W
// transposed (64 x 64, in x out) so that B[k = out][n = in] reads a row.
__device__ __forceinline__ void back64(const uint32_t a[4][4], const __nv_bfloat16 (*wt)[kLdW], const float h[8][4],
                                       float dz[8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma16816(acc, a[kk], ld2(&wt[8 * j + g][16 * kk + 2 * tig]), ld2(&wt[8 * j + g][16 * kk + 8 + 2 * tig]));
#pragma unroll
        for (int e = 0; e < 4; ++e) dz[j][e] = acc[e] * (1.0f - h[j][e] * h[j][e]);
    }
}

// Column sums over the warp's rows of a 16 x 64 accumulator-layout array
// into shared accumulators (one atomic per column and warp).
__device__ __forceinline__ void col_sums(const float v[8][4], float *dst) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const float s = rows_sum(v[j][e], v[j][e + 2]);
            if (g == 0) atomicAdd(&dst[8 * j + 2 * tig + e], s);
        }
}

// A 16 x 64 accumulator-layout array, BF16, into a transposed stage array
// (column c of the warp's local rows la, la + 8).
__device__ __forceinline__ void stage_t(const float v[8][4], __nv_bfloat16 (*dst)[kLdR], int la) {
    const int tig = threadIdx.x & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * tig;
        dst[c][la] = __float2bfloat16_rn(v[j][0]);
        dst[c + 1][la] = __float2bfloat16_rn(v[j][1]);
        dst[c][la + 8] = __float2bfloat16_rn(v[j][2]);
        dst[c + 1][la + 8] = __float2bfloat16_rn(v[j][3]);
    }
}

// Gradient of L = (1/N) Σ (y - t)² over n rows (N = n_total) into grad
// (FP32, accumulated with atomics) and Σ (y - t)² into loss. Each block
// step takes 128 rows: the 8 warps run forward and backward on 16 rows each
// in registers (mma.sync), stage the BF16 operands of the weight gradients
// transposed in shared memory, then each warp accumulates 9 of the 72
// 16 x 8 weight-gradient tiles (32 of dW3, 32 of dW2, 8 of dW1) over the
// step's 128 rows in registers, across the block's steps.
__global__ void __launch_bounds__(256, 1) k_mlp_grad(const float *__restrict__ p, const float *__restrict__ x,
                                                     const float *__restrict__ t, int64_t n, float two_over_n,
                                                     float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpWeights &S = *reinterpret_cast<MlpWeights *>(smem_raw);
    MlpStage &T = *reinterpret_cast<MlpStage *>(smem_raw + kWeightsBytes);
    stage_weights(p, S);
    for (int i = threadIdx.x; i < kH; i += blockDim.x) T.db1[i] = T.db2[i] = T.db3[i] = T.dw4[i] = 0.0f;
    if (threadIdx.x == 0) T.db4 = T.loss = 0.0f;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, tig = lane & 3;
    const int la = 16 * w + g, lb = la + 8;  // the thread's two rows within a block step
    float acc[9][4];
#pragma unroll
    for (int s = 0; s < 9; ++s) acc[s][0] = acc[s][1] = acc[s][2] = acc[s][3] = 0.0f;
    for (int64_t r0 = (int64_t)blockIdx.x * kRowsPerBlock; r0 < n; r0 += (int64_t)gridDim.x * kRowsPerBlock) {
        const int64_t ra = r0 + la, rb = r0 + lb;
        float xa[4], xb[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int f = 2 * tig + (q & 1) + 8 * (q >> 1);
            xa[q] = ra < n ? x[ra * kF + f] : 0.0f;
            xb[q] = rb < n ? x[rb * kF + f] : 0.0f;
            T.xt[f][la] = __float2bfloat16_rn(xa[q]);
            T.xt[f][lb] = __float2bfloat16_rn(xb[q]);
        }
        const uint32_t ax[4] = {pack2(xa[0], xa[1]), pack2(xb[0], xb[1]), pack2(xa[2], xa[3]), pack2(xb[2], xb[3])};
        WarpAct A;
        float y[2];
        warp_forward(S, ax, A, y);
        const float ea = ra < n ? y[0] - t[ra] : 0.0f, eb = rb < n ? y[1] - t[rb] : 0.0f;
        const float dya = ea * two_over_n, dyb = eb * two_over_n;
        // loss and db4: one count per row (tig == 0)
        const float l = rows_sum(tig == 0 ? ea * ea : 0.0f, tig == 0 ? eb * eb : 0.0f);
        const float d4 = rows_sum(tig == 0 ? dya : 0.0f, tig == 0 ? dyb : 0.0f);
        if (lane == 0) {
            atomicAdd(&T.loss, l);
            atomicAdd(&T.db4, d4);
        }
        // dZ3 = dy w4 (1 - h3²); dw4 += dy h3
        float dz[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float dy = e < 2 ? dya : dyb;
                dz[j][e] = dy * S.w4[8 * j + 2 * tig + (e & 1)] * (1.0f - A.h3[j][e] * A.h3[j][e]);
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float s4 = rows_sum(dya * A.h3[j][e], dyb * A.h3[j][e + 2]);
                if (g == 0) atomicAdd(&T.dw4[8 * j + 2 * tig + e], s4);
            }
        }
        col_sums(dz, T.db3);
        stage_t(dz, T.dz3t, la);
        stage_t(A.h2, T.h2t, la);
        uint32_t a[4][4];
        act_fragments(dz, a);
        back64(a, S.w3t, A.h2, dz);  // dZ2
        col_sums(dz, T.db2);
        stage_t(dz, T.dz2t, la);
        stage_t(A.h1, T.h1t, la);
        act_fragments(dz, a);
        back64(a, S.w2t, A.h1, dz);  // dZ1
        col_sums(dz, T.db1);
        stage_t(dz, T.dz1t, la);
        __syncthreads();
        // weight gradients over the step's 128 rows: warp w takes tiles
        // w + 8s (s < 4: dW3, s < 8: dW2, s = 8: dW1)
#pragma unroll
        for (int s = 0; s < 9; ++s) {
            const __nv_bfloat16(*Am)[kLdR] = s < 4 ? T.dz3t : (s < 8 ? T.dz2t : T.dz1t);
            const __nv_bfloat16(*Bm)[kLdR] = s < 4 ? T.h2t : (s < 8 ? T.h1t : T.xt);
            const int q = s < 8 ? w + 8 * (s & 3) : w;
            const int mt = s < 8 ? q >> 3 : q >> 1, nt = s < 8 ? q & 7 : q & 1;
#pragma unroll
            for (int kk = 0; kk < kRowsPerBlock / 16; ++kk) {
                const uint32_t af[4] = {ld2(&Am[16 * mt + g][16 * kk + 2 * tig]), ld2(&Am[16 * mt + g + 8][16 * kk + 2 * tig]),
                                        ld2(&Am[16 * mt + g][16 * kk + 8 + 2 * tig]),
                                        ld2(&Am[16 * mt + g + 8][16 * kk + 8 + 2 * tig])};
                mma16816(acc[s], af, ld2(&Bm[8 * nt + g][16 * kk + 2 * tig]), ld2(&Bm[8 * nt + g][16 * kk + 8 + 2 * tig]));
            }
        }
        __syncthreads();  // the next step overwrites the stage
    }
#pragma unroll
    for (int s = 0; s < 9; ++s) {
        const int q = s < 8 ? w + 8 * (s & 3) : w;
        const int mt = s < 8 ? q >> 3 : q >> 1, nt = s < 8 ? q & 7 : q & 1;
        const int base = s < 4 ? kOffW3 : (s < 8 ? kOffW2 : kOffW1), ld = s < 8 ? kH : kF;
        const int o = 16 * mt + g, i = 8 * nt + 2 * tig;
        atomicAdd(&grad[base + o * ld + i], acc[s][0]);
        atomicAdd(&grad[base + o * ld + i + 1], acc[s][1]);
        atomicAdd(&grad[base + (o + 8) * ld + i], acc[s][2]);
        atomicAdd(&grad[base + (o + 8) * ld + i + 1], acc[s][3]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        atomicAdd(&grad[kOffB1 + i], T.db1[i]);
        atomicAdd(&grad[kOffB2 + i], T.db2[i]);
        atomicAdd(&grad[kOffB3 + i], T.db3[i]);
        atomicAdd(&grad[kOffW4 + i], T.dw4[i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grad[kOffB4], T.db4);
        atomicAdd(loss, T.loss);
    }
}

// Adam on the FP32 master parameters; clears the gradient for the next step.
__global__ void k_mlp_adam(float *__restrict__ p, float *__restrict__ grad, float *__restrict__ m,
                           float *__restrict__ v, float lr, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float gr = grad[i];
    const float mm = 0.9f * m[i] + 0.1f * gr, vv = 0.999f * v[i] + 0.001f * gr * gr;
    m[i] = mm;
    v[i] = vv;
    p[i] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + 1e-8f);
    grad[i] = 0.0f;
}

// ------------------------------------------------------------------ features
constexpr double kKeplerGm = 3.986005e14;  // src/geometry/kepler.rs:12

// One transmitter's circular orbit: its raw elements (network inputs) and
// the constants of its position (CircularKeplerian, src/geometry/kepler.rs:
// 32-85: radius, mean motion, true anomaly at epoch, sines and cosines of
// inclination and RAAN, from the host's libm).
struct DevElem {
    double a, inc_deg, raan_deg, ta_deg;
    double r, mm, nu0, si, ci, so, co, epoch;
};

// Position and velocity (ECEF, m and m/s) of the orbit at e seconds after
// its epoch: the reference's expression and its time derivative.
__device__ __forceinline__ void elem_state(const DevElem &k, double e, double p[3], double v[3]) {
    const double nu = k.nu0 + k.mm * e;
    double snu, cnu;
    sincos(nu, &snu, &cnu);
    const double xp = k.r * cnu, yp = k.r * snu, dxp = -k.r * k.mm * snu, dyp = k.r * k.mm * cnu;
    const double y1 = yp * k.ci, z1 = yp * k.si, dy1 = dyp * k.ci, dz1 = dyp * k.si;
    const double xe = xp * k.co - y1 * k.so, ye = xp * k.so + y1 * k.co;
    const double dxe = dxp * k.co - dy1 * k.so, dye = dxp * k.so + dy1 * k.co;
    double s, c;
    sincos(kEarthRate * e, &s, &c);
    p[0] = xe * c + ye * s;
    p[1] = -xe * s + ye * c;
    p[2] = z1;
    v[0] = dxe * c + dye * s + kEarthRate * p[1];
    v[1] = -dxe * s + dye * c - kEarthRate * p[0];
    v[2] = dz1;
}

// The 16 raw features of (orbit, receiver O, reception time t, scene
// epoch): the elements, O, t, then from the orbit at t: the line-of-sight
// unit vector, R/c, range rate / c, v_x / c, v_y / c and the Sagnac rate of
// the line of sight. R: the orbit's range at t (m).
__device__ __forceinline__ void elem_features(const DevElem &k, double ox, double oy, double oz, double epoch,
                                              double t, float f[kF], double &R) {
    double p[3], v[3];
    elem_state(k, (epoch - k.epoch) + t, p, v);
    const double dx = p[0] - ox, dy = p[1] - oy, dz = p[2] - oz;
    R = sqrt(dx * dx + dy * dy + dz * dz);
    const double inv = R > 0.0 ? 1.0 / R : 0.0, ic = 1.0 / kSpeedOfLight;
    const double ux = dx * inv, uy = dy * inv, uz = dz * inv;
    f[0] = (float)k.a;
    f[1] = (float)k.inc_deg;
    f[2] = (float)k.raan_deg;
    f[3] = (float)k.ta_deg;
    f[4] = (float)ox;
    f[5] = (float)oy;
    f[6] = (float)oz;
    f[7] = (float)t;
    f[8] = (float)ux;
    f[9] = (float)uy;
    f[10] = (float)uz;
    f[11] = (float)(R * ic);
    f[12] = (float)((v[0] * ux + v[1] * uy + v[2] * uz) * ic);
    f[13] = (float)(v[0] * ic);
    f[14] = (float)(v[1] * ic);
    f[15] = (float)(kEarthRate * (p[0] * oy - p[1] * ox) * inv * ic);
}

// ------------------------------------------------------------------ solver
// Geometric range at the reception time tu (trajectory table on its natural
// segment, query time unrounded).
__device__ __forceinline__ double table_range(const DevTx &tx, double tu, double de, double ox, double oy,
                                              double oz) {
    bool cl;
    const int64_t lo = seg_unrounded(tx, tu, de, cl);
    double px, py, pz;
    pos_unrounded(tx, tu, de, lo, px, py, pz);
    const double dx = px - ox, dy = py - oy, dz = pz - oz;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Converged light-time solve of delay τ from the start `tau`, on the same
// model as the reference (lerp table, linearised Sagnac ω·τ), with the query
// time unrounded. FIXED_POINT iterates the reference's map τ <- R(tu-τ)/c;
// NEWTON divides its residual by 1 - dR/dτ / c. Returns the number of map
// evaluations, or -1 when |Δτ| stayed above tol for max_iter evaluations.
__device__ int converge(const DevTx &tx, double tu, double de, double ox, double oy, double oz, double tol,
                        int max_iter, int scheme, double tau, double &out) {
    for (int it = 1; it <= max_iter; ++it) {
        const double tq = tu - tau;
        bool cl;
        const int64_t lo = seg_unrounded(tx, tq, de, cl);
        double px, py, pz;
        pos_unrounded(tx, tq, de, lo, px, py, pz);
        const double w = kEarthRate * tau;
        const double dx = px + w * py - ox, dy = py - w * px - oy, dz = pz - oz;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double gv = r / kSpeedOfLight;
        double tn = gv;
        if (scheme == 1) {
            double vx = 0.0, vy = 0.0, vz = 0.0;
            if (tx.traj_kind != 0) {
                const double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
                vx = (b.x - a.x) / tx.dt;
                vy = (b.y - a.y) / tx.dt;
                vz = (b.z - a.z) / tx.dt;
            }
            const double ddx = -vx + kEarthRate * py - w * vy, ddy = -vy - kEarthRate * px + w * vx, ddz = -vz;
            const double gp = (dx * ddx + dy * ddy + dz * ddz) / (r * kSpeedOfLight);
            tn = tau - (tau - gv) / (1.0 - gp);
        }
        if (fabs(tn - tau) <= tol) {
            out = tn;
            return it;
        }
        tau = tn;
    }
    out = tau;
    return -1;
}

constexpr double kLagStart = 0.07;  // the reference's initial guess, src/channel/mod.rs:23

// One thread per sample: start, converge, fall back to the LAG start when a
// GEOMETRIC / LEARNED start does not converge. Sample i solves transmitter
// tx_idx[i] (or tx_const) for receiver rx3[rx_idx[i]] (or rx3[0]); the
// learned start is base[i] (the orbit's R/c) plus the network's
// de-normalised correction pred[i] (µs).
__global__ void __launch_bounds__(128)
k_solve_converged(const DevTx *__restrict__ txs, const int32_t *__restrict__ tx_idx, int32_t tx_const,
                  const double *__restrict__ rx3, const int32_t *__restrict__ rx_idx, double epoch,
                  const double *__restrict__ tu, int64_t n, double tol, int32_t max_iter, int32_t scheme,
                  int32_t start, const double *__restrict__ base, const float *__restrict__ pred, float tmean,
                  float tstd, double *__restrict__ temit, int32_t *__restrict__ iters, float *__restrict__ start_err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevTx &tx = txs[tx_idx ? tx_idx[i] : tx_const];
    const int r = rx_idx ? rx_idx[i] : 0;
    const double ox = rx3[3 * r], oy = rx3[3 * r + 1], oz = rx3[3 * r + 2];
    const double de = tx.traj_kind != 0 ? epoch - tx.t0 : 0.0;
    const double t = tu[i];
    double tau0 = kLagStart;
    if (start == 1) tau0 = table_range(tx, t, de, ox, oy, oz) / kSpeedOfLight;
    if (start == 2) tau0 = base[i] + (double)fmaf(pred[i], tstd, tmean) * 1e-6;  // correction in µs
    double tau;
    int it = converge(tx, t, de, ox, oy, oz, tol, max_iter, scheme, tau0, tau);
    if (it < 0 && start != 0) {
        int it2 = converge(tx, t, de, ox, oy, oz, tol, max_iter, scheme, kLagStart, tau);
        it = it2 < 0 ? -1 : max_iter + it2;
    }
    temit[i] = t - tau;
    iters[i] = it;
    if (start_err) start_err[i] = (float)fabs(tau0 - tau);
}

// Features of n samples (normalised when norm is given) and the orbit's
// R/c at each (the learned start's base). Sample i: orbit k_of_tx[tx_idx[i]]
// (or of tx_const), receiver rx3[rx_idx[i]] (or rx3[0]).
__global__ void __launch_bounds__(128)
k_elem_features(const DevElem *__restrict__ el, const int32_t *__restrict__ k_of_tx, const int32_t *__restrict__ tx_idx,
                int32_t tx_const, const double *__restrict__ rx3, const int32_t *__restrict__ rx_idx, double epoch,
                const double *__restrict__ tu, int64_t n, const float *__restrict__ norm, float *__restrict__ x,
                double *__restrict__ base) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = k_of_tx[tx_idx ? tx_idx[i] : tx_const];
    const int r = rx_idx ? rx_idx[i] : 0;
    float f[kF];
    double R;
    elem_features(el[k], rx3[3 * r], rx3[3 * r + 1], rx3[3 * r + 2], epoch, tu[i], f, R);
#pragma unroll
    for (int q = 0; q < kF; ++q) x[i * kF + q] = norm ? (f[q] - norm[q]) / norm[kF + q] : f[q];
    if (base) base[i] = R / kSpeedOfLight;
}

// Training set: sample i draws (from Philox counter i, tag "MLPT") an orbit
// k, a receiver j and a reception time uniform in [t0, t1); its raw
// features and the light-time correction τ - R_orbit/c (µs) of the
// converged Newton solve (tolerance 1e-16 s) on transmitter scene_tx[k]'s
// trajectory table, started at R_orbit/c.
__global__ void __launch_bounds__(128)
k_mlp_dataset(const DevTx *__restrict__ txs, const int32_t *__restrict__ scene_tx, const DevElem *__restrict__ el,
              int32_t n_el, const double *__restrict__ rx3, int32_t n_rx, double epoch, double t0, double t1, int64_t n,
              uint64_t seed, float *__restrict__ x, float *__restrict__ y, int32_t *__restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 rr = philox4x32_10(make_uint4((uint32_t)(uint64_t)i, (uint32_t)((uint64_t)i >> 32), 0x4D4C5054u, 0u),
                                   make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double u = (double)(((uint64_t)rr.x << 21) ^ (uint64_t)(rr.y >> 11)) * 0x1.0p-53;
    const double t = t0 + (t1 - t0) * u;
    const int k = (int)__umulhi(rr.z, (uint32_t)n_el), j = (int)__umulhi(rr.w, (uint32_t)n_rx);
    const DevTx &tx = txs[scene_tx[k]];
    const double ox = rx3[3 * j], oy = rx3[3 * j + 1], oz = rx3[3 * j + 2];
    float f[kF];
    double R, tau;
    elem_features(el[k], ox, oy, oz, epoch, t, f, R);
    const double de = tx.traj_kind != 0 ? epoch - tx.t0 : 0.0;
    const int it = converge(tx, t, de, ox, oy, oz, 1e-16, 20, 1, R / kSpeedOfLight, tau);
    if (it < 0) atomicAdd(bad, 1);
#pragma unroll
    for (int q = 0; q < kF; ++q) x[i * kF + q] = f[q];
    y[i] = (float)((tau - R / kSpeedOfLight) * 1e6);
}

__global__ void k_mlp_normalize(float *__restrict__ x, float *__restrict__ y, int64_t n,
                                const float *__restrict__ norm) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int k = 0; k < kF; ++k) x[i * kF + k] = (x[i * kF + k] - norm[k]) / norm[kF + k];
    y[i] = (y[i] - norm[2 * kF]) / norm[2 * kF + 1];
}

// ---------------------------------------------------------------------------
// Forward pass on the 5th-generation tensor cores (inference: lpk_mlp_forward
// and the learned start of the converged solve). One CTA of 4 warps takes
// tiles of 128 rows: the tile's inputs and hidden layers are staged in shared
// memory in the no-swizzle K-major core-matrix layout that tcgen05.mma reads
// (8 rows x 16 bytes per core matrix; next 8-row group +128 B, next 8
// K-elements +rows*16 B), one thread issues the MMAs (M = 128, N = 64,
// K = 16 per instruction, BF16 operands, FP32 accumulator in TMEM), commits
// them to an mbarrier, and each warp reads its 32 rows of the accumulator
// back with tcgen05.ld for the tanh epilogue. Rounding points are those of
// the mma.sync training kernel (BF16 x, W1-W3 and the first two hidden
// layers; FP32 accumulation and everything else), so the CPU restatement
// covers both; only the FP32 summation order differs (bias added after the
// products).
constexpr int kTcRows = 128;          // rows per tile = the MMA's M
constexpr uint32_t kTcCols = 64;      // TMEM columns: one 128 x 64 FP32 accumulator, reused by every layer
// kind::f16 instruction descriptor: FP32 accumulator (bits 4-5 = 1), BF16 A
// (7-9 = 1) and B (10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kH >> 3) << 17) |
                              ((uint32_t)(kTcRows >> 4) << 24);
constexpr int kTcSpin = 1 << 20;      // mbarrier polls before a wait gives up

struct __align__(1024) TcSmem {
    __nv_bfloat16 a1[2][kTcRows][8];       // x tile: features 0-7 and 8-15
    __nv_bfloat16 a2[kH / 8][kTcRows][8];  // a hidden layer (the first, then the second), 8 column groups
    __nv_bfloat16 b1[2][kH][8];            // W1 (out x in)
    __nv_bfloat16 b2[kH / 8][kH][8];       // W2 (out x in)
    __nv_bfloat16 b3[kH / 8][kH][8];       // W3 (out x in)
    float bias1[kH], bias2[kH], bias3[kH], w4[kH];
    float b4;
    unsigned long long bar;
    uint32_t tmem;
};
// At most 5 CTAs of this size fit on an SM (228 KB), so their TMEM demand
// (5 x 64 columns) stays within the SM's 512 and tcgen05.alloc never waits
// on another CTA.
static_assert((228 * 1024 / sizeof(TcSmem)) * kTcCols <= 512, "TMEM residency bound");

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle, K-major): start address,
// leading byte offset (next 8 K-elements), stride byte offset (next 8 rows),
// all in 16-byte units; version 1 (bit 46); base offset, LBO mode and layout
// type 0.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate,
                                       uint32_t idesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Poll the mbarrier's phase at most `spin` times; false when it never flipped.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase, int spin) {
    for (int it = 0; it < spin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// This warp's 32 accumulator rows (lane = row), 64 FP32 columns.
__device__ __forceinline__ void tc_load_row(uint32_t taddr, float v[kH]) {
#pragma unroll
    for (int q = 0; q < kH / 16; ++q) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr + (uint32_t)(16 * q)));
#pragma unroll
        for (int i = 0; i < 16; ++i) v[16 * q + i] = __uint_as_float(r[i]);
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// tanh(h + bias) of this thread's row, BF16, into the row of a hidden tile.
__device__ __forceinline__ void tc_store_hidden(const float h[kH], const float *bias, __nv_bfloat16 (*dst)[kTcRows][8],
                                                int row) {
#pragma unroll
    for (int g = 0; g < kH / 8; ++g) {
        uint4 pk;
        pk.x = pack2(tanhf(h[8 * g + 0] + bias[8 * g + 0]), tanhf(h[8 * g + 1] + bias[8 * g + 1]));
        pk.y = pack2(tanhf(h[8 * g + 2] + bias[8 * g + 2]), tanhf(h[8 * g + 3] + bias[8 * g + 3]));
        pk.z = pack2(tanhf(h[8 * g + 4] + bias[8 * g + 4]), tanhf(h[8 * g + 5] + bias[8 * g + 5]));
        pk.w = pack2(tanhf(h[8 * g + 6] + bias[8 * g + 6]), tanhf(h[8 * g + 7] + bias[8 * g + 7]));
        *reinterpret_cast<uint4 *>(&dst[g][row][0]) = pk;
    }
}

// y = MLP(x) for n rows of normalised features. err (may be NULL) gets 1 if
// an MMA completion wait gave up after `spin` polls (the outputs are then
// incomplete). withhold (self-test only) issues no MMA and no commit, so
// every wait runs out with nothing in flight. A wait that gives up on a
// real MMA leaves the loop and deallocates the TMEM with that MMA possibly
// still in flight: the alternative, keeping the columns, would leave every
// later CTA on this SM waiting in tcgen05.alloc.
__global__ void __launch_bounds__(128, 1) k_mlp_forward_tc(const float *__restrict__ p, const float *__restrict__ x,
                                                           int64_t n, float *__restrict__ y, int *__restrict__ err,
                                                           int spin, int withhold) {
    __shared__ TcSmem S;
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights in the core-matrix layout, biases
    for (int i = tid; i < 2 * kH * 8; i += blockDim.x) {
        const int g = i / (kH * 8), o = (i / 8) % kH, c = i % 8;
        S.b1[g][o][c] = __float2bfloat16_rn(p[kOffW1 + o * kF + 8 * g + c]);
    }
    for (int i = tid; i < kH * kH; i += blockDim.x) {
        const int o = i / kH, k = i % kH;
        S.b2[k / 8][o][k % 8] = __float2bfloat16_rn(p[kOffW2 + i]);
        S.b3[k / 8][o][k % 8] = __float2bfloat16_rn(p[kOffW3 + i]);
    }
    for (int i = tid; i < kH; i += blockDim.x) {
        S.bias1[i] = p[kOffB1 + i];
        S.bias2[i] = p[kOffB2 + i];
        S.bias3[i] = p[kOffB3 + i];
        S.w4[i] = p[kOffW4 + i];
    }
    if (tid == 0) {
        S.b4 = p[kOffB4];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem, bar = smem_u32(&S.bar);
    const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);  // this warp's lane quarter
    const uint64_t d_a1 = tc_desc(smem_u32(&S.a1[0][0][0]), kTcRows * 16, 128);
    const uint64_t d_b1 = tc_desc(smem_u32(&S.b1[0][0][0]), kH * 16, 128);
    uint32_t phase = 0;
    bool ok = true;
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int64_t row = t * kTcRows + tid;
        // inputs of this thread's row, BF16, into the two column groups of the tile
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            float v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = row < n ? x[row * kF + 8 * g + k] : 0.0f;
            uint4 pk;
            pk.x = pack2(v[0], v[1]);
            pk.y = pack2(v[2], v[3]);
            pk.z = pack2(v[4], v[5]);
            pk.w = pack2(v[6], v[7]);
            *reinterpret_cast<uint4 *>(&S.a1[g][tid][0]) = pk;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> the MMA's reads
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !withhold) {
            tc_fence_after();
            tc_mma(tmem, d_a1, d_b1, 0u, kTcIdesc);  // layer 1: one K = 16 step
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase, spin));
        phase ^= 1u;
        if (!ok) break;
        float h[kH];
#pragma unroll
        for (int layer = 2; layer <= 3; ++layer) {
            tc_fence_after();
            tc_load_row(trow, h);
            tc_store_hidden(h, layer == 2 ? S.bias1 : S.bias2, S.a2, tid);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncthreads();  // every warp has read the accumulator and written its rows
            if (tid == 0 && !withhold) {
                tc_fence_after();
                const __nv_bfloat16(*w)[kH][8] = layer == 2 ? S.b2 : S.b3;
#pragma unroll
                for (int kk = 0; kk < kH / 16; ++kk)  // four K = 16 steps
                    tc_mma(tmem, tc_desc(smem_u32(&S.a2[2 * kk][0][0]), kTcRows * 16, 128),
                           tc_desc(smem_u32(&w[2 * kk][0][0]), kH * 16, 128), kk > 0 ? 1u : 0u, kTcIdesc);
                tc_commit(bar);
            }
            ok = __syncthreads_and(tc_wait(bar, phase, spin));
            phase ^= 1u;
            if (!ok) break;
        }
        if (!ok) break;
        tc_fence_after();
        tc_load_row(trow, h);
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < kH; ++c) s = fmaf(tanhf(h[c] + S.bias3[c]), S.w4[c], s);
        if (row < n) y[row] = s + S.b4;
        tc_fence_before();
        __syncthreads();  // the tiles and the accumulator are reused by the next tile
        tc_fence_after();
    }
    if (!ok && tid == 0 && err) atomicOr(err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
    }
}

// The tensor-core forward over n rows on `st`; d_err: one int of device memory.
cudaError_t launch_mlp_forward(const float *d_p, const float *d_x, int64_t n, float *d_y, int *d_err, int sms,
                               cudaStream_t st, int spin = kTcSpin, int withhold = 0) {
    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (e != cudaSuccess || n <= 0) return e;
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    // five CTAs per SM: what shared memory allows (and 5 x 64 TMEM columns fit)
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 5 * (int64_t)sms));
    k_mlp_forward_tc<<<grid, 128, 0, st>>>(d_p, d_x, n, d_y, d_err, spin, withhold);
    return cudaGetLastError();
}

inline double deg2rad(double deg) { return deg * (M_PI / 180.0); }  // f64::to_radians

}  // namespace
}  // namespace lpk

using namespace lpk;

struct lpk_mlp {
    lpk_ctx *ctx = nullptr;
    float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr, *d_norm = nullptr;
    int *d_err = nullptr;  // set by the inference kernel when a tensor-core completion wait gives up
    float norm[kNorm];     // feature means, feature stds, target mean, target std (µs)
    int64_t step = 0;
    // the scene's orbits: the network's transmitters, their elements, and
    // for every uploaded transmitter its orbit index (-1: not in the set)
    std::vector<int32_t> k_of_tx;
    std::vector<int32_t> scene_tx;
    DevElem *d_el = nullptr;
    int32_t *d_k_of_tx = nullptr, *d_scene_tx = nullptr;
};

namespace {

lpk_status upload(lpk_ctx *c, void *dst, const void *src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "upload");
}

lpk_status launch_grad(lpk_mlp *m, const float *d_x, const float *d_t, int64_t n, float *d_loss) {
    lpk_ctx *c = m->ctx;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp gradient shared memory");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int64_t steps = (n + kRowsPerBlock - 1) / kRowsPerBlock;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(steps, sms));
    k_mlp_grad<<<grid, 256, kGradSmem, c->stream>>>(m->d_p, d_x, d_t, n, 2.0f / (float)n, m->d_g, d_loss);
    e = cudaGetLastError();
    c->launches += 1;
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "mlp gradient kernel");
}

void free_orbits(lpk_mlp *m) {
    for (void *p : {(void *)m->d_el, (void *)m->d_k_of_tx, (void *)m->d_scene_tx})
        if (p) cudaFree(p);
    m->d_el = nullptr;
    m->d_k_of_tx = m->d_scene_tx = nullptr;
    m->k_of_tx.clear();
    m->scene_tx.clear();
}

// Set the network's orbits (lpk_mlp_set_orbits' body).
lpk_status set_orbits(lpk_mlp *m, const int32_t *tx, const lpk_kepler_orbit *orbits, int32_t n_tx) {
    lpk_ctx *c = m->ctx;
    if (n_tx < 1 || !tx || !orbits) return fail(c, LPK_EINVAL, "the network needs at least one transmitter orbit");
    std::vector<int32_t> k_of(c->n_tx, -1);
    std::vector<DevElem> el((size_t)n_tx);
    for (int32_t k = 0; k < n_tx; ++k) {
        if (tx[k] < 0 || tx[k] >= c->n_tx) return fail(c, LPK_EINVAL, "transmitter index out of range of the scene");
        if (k_of[tx[k]] >= 0) return fail(c, LPK_EINVAL, "a transmitter appears twice in the network's orbits");
        if (c->h_tx[tx[k]].traj_kind == 0) return fail(c, LPK_EINVAL, "the network's transmitters must move");
        k_of[tx[k]] = k;
        const lpk_kepler_orbit &o = orbits[k];
        const double r = o.semi_major_axis_m;
        if (!(r > 0.0) || !std::isfinite(r) || !std::isfinite(o.epoch_unix))
            return fail(c, LPK_EINVAL, "orbit elements must be finite with a positive semi-major axis");
        const double inc = deg2rad(o.inclination_deg), om = deg2rad(o.raan_deg);
        el[k] = DevElem{r, o.inclination_deg, o.raan_deg, o.true_anomaly_deg_at_epoch,
                        r, std::sqrt(kKeplerGm / (r * r * r)), deg2rad(o.true_anomaly_deg_at_epoch),
                        std::sin(inc), std::cos(inc), std::sin(om), std::cos(om), o.epoch_unix};
    }
    free_orbits(m);
    if (cudaMalloc((void **)&m->d_el, sizeof(DevElem) * el.size()) != cudaSuccess ||
        cudaMalloc((void **)&m->d_k_of_tx, sizeof(int32_t) * (size_t)std::max(c->n_tx, 1)) != cudaSuccess ||
        cudaMalloc((void **)&m->d_scene_tx, sizeof(int32_t) * (size_t)n_tx) != cudaSuccess) {
        free_orbits(m);
        return fail(c, LPK_ENOMEM, "mlp orbit table allocation failed");
    }
    m->k_of_tx = k_of;
    m->scene_tx.assign(tx, tx + n_tx);
    lpk_status s = upload(c, m->d_el, el.data(), sizeof(DevElem) * el.size());
    if (!s && c->n_tx > 0) s = upload(c, m->d_k_of_tx, k_of.data(), sizeof(int32_t) * k_of.size());
    if (!s) s = upload(c, m->d_scene_tx, tx, sizeof(int32_t) * (size_t)n_tx);
    if (!s && cudaStreamSynchronize(c->stream) != cudaSuccess) s = fail(c, LPK_ECUDA, "mlp orbit upload");
    return s;
}

// The converged solve behind lpk_solve_converged and lpk_solve_converged_scene:
// sample i solves transmitter tx_idx[i] (tx_const when tx_idx is NULL) for
// receiver rx3[rx_idx[i]] (rx3[0] when rx_idx is NULL). Host memory in and
// out; device_ms (may be NULL) gets the device time of the call's kernels.
lpk_status solve_impl(lpk_ctx *c, const int32_t *tx_idx, int32_t tx_const, const double *rx3, const int32_t *rx_idx,
                      int32_t n_rx, double epoch, const double *t_rel_utc, int64_t n, double tol_s, int32_t max_iter,
                      int32_t scheme, int32_t start, const lpk_mlp *m, double *t_emit, int32_t *iters,
                      float *start_err, double *device_ms) {
    if (n < 0 || (n > 0 && (!t_rel_utc || !t_emit || !iters))) return fail(c, LPK_EINVAL, "bad solve arguments");
    if (!rx3 || n_rx < 1) return fail(c, LPK_EINVAL, "rx_ecef is NULL");
    if (scheme != LPK_ITER_FIXED_POINT && scheme != LPK_ITER_NEWTON) return fail(c, LPK_EINVAL, "unknown scheme");
    if (start != LPK_START_LAG && start != LPK_START_GEOMETRIC && start != LPK_START_LEARNED)
        return fail(c, LPK_EINVAL, "unknown start");
    if (start == LPK_START_LEARNED && (!m || m->ctx != c || m->scene_tx.empty()))
        return fail(c, LPK_EINVAL, "learned start needs a trained mlp of this context");
    if (!(tol_s >= 0.0) || max_iter < 1) return fail(c, LPK_EINVAL, "tol must be >= 0 and max_iter >= 1");
    for (int64_t i = 0; i < (tx_idx ? n : 1); ++i) {
        const int32_t tx = tx_idx ? tx_idx[i] : tx_const;
        if (tx < 0 || tx >= c->n_tx) return fail(c, LPK_EINVAL, "transmitter index out of range of the uploaded scene");
        if (start == LPK_START_LEARNED && ((size_t)tx >= m->k_of_tx.size() || m->k_of_tx[tx] < 0))
            return fail(c, LPK_EINVAL, "learned start: transmitter is not among the network's orbits");
    }
    if (rx_idx)
        for (int64_t i = 0; i < n; ++i)
            if (rx_idx[i] < 0 || rx_idx[i] >= n_rx) return fail(c, LPK_EINVAL, "receiver index out of range");
    if (device_ms) *device_ms = 0.0;
    if (n == 0) return LPK_OK;
    cudaSetDevice(c->device);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const bool learned = start == LPK_START_LEARNED;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += al(b); return o; };
    const size_t o_t = take(sizeof(double) * (size_t)n), o_o = take(sizeof(double) * (size_t)n);
    const size_t o_i = take(sizeof(int32_t) * (size_t)n), o_e = take(sizeof(float) * (size_t)n);
    const size_t o_tx = tx_idx ? take(sizeof(int32_t) * (size_t)n) : 0, o_rx = rx_idx ? take(sizeof(int32_t) * (size_t)n) : 0;
    const size_t o_r3 = take(sizeof(double) * 3 * (size_t)n_rx);
    const size_t o_x = learned ? take(sizeof(float) * (size_t)n * kF) : 0;
    const size_t o_p = learned ? take(sizeof(float) * (size_t)n) : 0, o_b = learned ? take(sizeof(double) * (size_t)n) : 0;
    const size_t o_err = take(sizeof(int));
    lpk_status s = ensure_scratch(c, off);
    if (s) return s;
    char *base = (char *)c->d_scratch;
    double *d_t = (double *)(base + o_t), *d_o = (double *)(base + o_o), *d_r3 = (double *)(base + o_r3);
    int32_t *d_i = (int32_t *)(base + o_i), *d_tx = tx_idx ? (int32_t *)(base + o_tx) : nullptr;
    int32_t *d_rx = rx_idx ? (int32_t *)(base + o_rx) : nullptr;
    float *d_e = (float *)(base + o_e), *d_x = (float *)(base + o_x), *d_p = (float *)(base + o_p);
    double *d_b = (double *)(base + o_b);
    int *d_err = (int *)(base + o_err);
    if ((s = upload(c, d_t, t_rel_utc, sizeof(double) * (size_t)n))) return s;
    if ((s = upload(c, d_r3, rx3, sizeof(double) * 3 * (size_t)n_rx))) return s;
    if (d_tx && (s = upload(c, d_tx, tx_idx, sizeof(int32_t) * (size_t)n))) return s;
    if (d_rx && (s = upload(c, d_rx, rx_idx, sizeof(int32_t) * (size_t)n))) return s;
    cudaEventRecord(c->ev_start, c->stream);
    const unsigned grid = (unsigned)((n + 127) / 128);
    if (learned) {
        k_elem_features<<<grid, 128, 0, c->stream>>>(m->d_el, m->d_k_of_tx, d_tx, tx_const, d_r3, d_rx, epoch, d_t, n,
                                                     m->d_norm, d_x, d_b);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        cudaError_t fe = launch_mlp_forward(m->d_p, d_x, n, d_p, d_err, sms, c->stream);
        if (fe != cudaSuccess) return cuda_fail(c, fe, "mlp forward");
        c->launches += 2;
    }
    k_solve_converged<<<grid, 128, 0, c->stream>>>(c->d_tx, d_tx, tx_const, d_r3, d_rx, epoch, d_t, n, tol_s,
                                                   max_iter, scheme, start, d_b, d_p, m ? m->norm[2 * kF] : 0.0f,
                                                   m ? m->norm[2 * kF + 1] : 1.0f, d_o, d_i, start_err ? d_e : nullptr);
    c->launches += 1;
    cudaEventRecord(c->ev_stop, c->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(t_emit, d_o, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(iters, d_i, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && start_err)
        e = cudaMemcpyAsync(start_err, d_e, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    int herr = 0;
    if (e == cudaSuccess && learned) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "converged solve");
    if (device_ms) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev_start, c->ev_stop);
        *device_ms = ms;
    }
    return herr ? fail(c, LPK_ETIMEDOUT, "learned start: a tensor-core completion wait gave up") : LPK_OK;
}

}  // namespace

extern "C" {

lpk_status lpk_mlp_create(lpk_ctx *c, uint64_t seed, lpk_mlp **out) {
    if (!c || !out) return fail(c, LPK_EINVAL, "NULL argument");
    *out = nullptr;
    cudaSetDevice(c->device);
    lpk_mlp *m = new lpk_mlp();
    m->ctx = c;
    float **bufs[5] = {&m->d_p, &m->d_m, &m->d_v, &m->d_g, &m->d_norm};
    for (int k = 0; k < 5; ++k) {
        cudaError_t e = cudaMalloc((void **)bufs[k], sizeof(float) * (k == 4 ? kNorm : kParams));
        if (e != cudaSuccess) {
            lpk_mlp_destroy(m);
            return fail(c, LPK_ENOMEM, "mlp allocation failed");
        }
    }
    if (cudaMalloc((void **)&m->d_err, sizeof(int)) != cudaSuccess ||
        cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess) {
        lpk_mlp_destroy(m);
        return fail(c, LPK_ENOMEM, "mlp allocation failed");
    }
    // Glorot-uniform weights from a SplitMix64 stream, zero biases
    std::vector<float> p(kParams, 0.0f);
    uint64_t st = seed;
    auto uni = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
    };
    const double a1 = std::sqrt(6.0 / (kF + kH)), a2 = std::sqrt(6.0 / (kH + kH)), a4 = std::sqrt(6.0 / (kH + 1));
    for (int i = 0; i < kH * kF; ++i) p[kOffW1 + i] = (float)(a1 * uni());
    for (int i = 0; i < kH * kH; ++i) p[kOffW2 + i] = (float)(a2 * uni());
    for (int i = 0; i < kH * kH; ++i) p[kOffW3 + i] = (float)(a2 * uni());
    for (int i = 0; i < kH; ++i) p[kOffW4 + i] = (float)(a4 * uni());
    for (int k = 0; k < kF; ++k) {
        m->norm[k] = 0.0f;
        m->norm[kF + k] = 1.0f;
    }
    m->norm[2 * kF] = 0.0f;
    m->norm[2 * kF + 1] = 1.0f;
    lpk_status s = upload(c, m->d_p, p.data(), sizeof(float) * kParams);
    if (!s) s = upload(c, m->d_norm, m->norm, sizeof m->norm);
    if (!s && (cudaMemsetAsync(m->d_m, 0, sizeof(float) * kParams, c->stream) != cudaSuccess ||
               cudaMemsetAsync(m->d_v, 0, sizeof(float) * kParams, c->stream) != cudaSuccess ||
               cudaMemsetAsync(m->d_g, 0, sizeof(float) * kParams, c->stream) != cudaSuccess))
        s = fail(c, LPK_ECUDA, "mlp state reset failed");
    if (!s && cudaStreamSynchronize(c->stream) != cudaSuccess) s = fail(c, LPK_ECUDA, "mlp create synchronize");
    if (s) {
        lpk_mlp_destroy(m);
        return s;
    }
    *out = m;
    return LPK_OK;
}

void lpk_mlp_destroy(lpk_mlp *m) {
    if (!m) return;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    for (float *p : {m->d_p, m->d_m, m->d_v, m->d_g, m->d_norm})
        if (p) cudaFree(p);
    if (m->d_err) cudaFree(m->d_err);
    free_orbits(m);
    delete m;
}

lpk_status lpk_mlp_get_params(const lpk_mlp *m, float *params, float *norm) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    cudaSetDevice(c->device);
    if (params) {
        cudaError_t e = cudaMemcpyAsync(params, m->d_p, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "mlp parameter read");
    }
    if (norm) memcpy(norm, m->norm, sizeof m->norm);
    return LPK_OK;
}

lpk_status lpk_mlp_set_params(lpk_mlp *m, const float *params, const float *norm) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    cudaSetDevice(c->device);
    lpk_status s = LPK_OK;
    if (params) s = upload(c, m->d_p, params, sizeof(float) * kParams);
    if (!s && norm) {
        for (int k = 0; k < kF; ++k)
            if (!(norm[kF + k] > 0.0f)) return fail(c, LPK_EINVAL, "normalisation stds must be positive");
        if (!(norm[2 * kF + 1] > 0.0f)) return fail(c, LPK_EINVAL, "normalisation stds must be positive");
        memcpy(m->norm, norm, sizeof m->norm);
        s = upload(c, m->d_norm, m->norm, sizeof m->norm);
    }
    if (!s && cudaStreamSynchronize(c->stream) != cudaSuccess) s = fail(c, LPK_ECUDA, "mlp parameter write");
    return s;
}

lpk_status lpk_mlp_set_orbits(lpk_mlp *m, const int32_t *tx, const lpk_kepler_orbit *orbits, int32_t n_tx) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    cudaSetDevice(m->ctx->device);
    return set_orbits(m, tx, orbits, n_tx);
}

lpk_status lpk_mlp_forward(lpk_mlp *m, const float *x, int64_t n, float *y) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    if (n < 0 || (n > 0 && (!x || !y))) return fail(c, LPK_EINVAL, "bad forward arguments");
    if (n == 0) return LPK_OK;
    cudaSetDevice(c->device);
    const size_t bx = sizeof(float) * (size_t)n * kF, by = sizeof(float) * (size_t)n;
    const size_t oy = (bx + 255) / 256 * 256, oe = oy + (by + 255) / 256 * 256;
    lpk_status s = ensure_scratch(c, oe + 256);
    if (s) return s;
    float *d_x = (float *)c->d_scratch, *d_y = (float *)((char *)c->d_scratch + oy);
    int *d_err = (int *)((char *)c->d_scratch + oe);
    if ((s = upload(c, d_x, x, bx))) return s;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    cudaError_t e = launch_mlp_forward(m->d_p, d_x, n, d_y, d_err, sms, c->stream);
    c->launches += 1;
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, d_y, by, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp forward");
    return herr ? fail(c, LPK_ETIMEDOUT, "mlp forward: a tensor-core completion wait gave up") : LPK_OK;
}

lpk_status lpk_mlp_wait_selftest(lpk_mlp *m, int64_t n, int32_t spin) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    if (n < 1 || spin < 1) return fail(c, LPK_EINVAL, "self-test needs n >= 1 and spin >= 1");
    cudaSetDevice(c->device);
    const size_t bx = sizeof(float) * (size_t)n * kF, by = sizeof(float) * (size_t)n;
    const size_t oy = (bx + 255) / 256 * 256, oe = oy + (by + 255) / 256 * 256;
    lpk_status s = ensure_scratch(c, oe + 256);
    if (s) return s;
    float *d_x = (float *)c->d_scratch, *d_y = (float *)((char *)c->d_scratch + oy);
    int *d_err = (int *)((char *)c->d_scratch + oe);
    cudaError_t e = cudaMemsetAsync(d_x, 0, bx, c->stream);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e == cudaSuccess) e = launch_mlp_forward(m->d_p, d_x, n, d_y, d_err, sms, c->stream, spin, 1);
    c->launches += 1;
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp wait self-test");
    return herr ? fail(c, LPK_ETIMEDOUT, "mlp wait self-test: every tensor-core completion wait gave up, as withheld")
                : fail(c, LPK_EINVAL, "mlp wait self-test: a withheld wait did not give up");
}

lpk_status lpk_mlp_loss_grad(lpk_mlp *m, const float *x, const float *t, int64_t n, double *loss, float *grad) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    if (n <= 0 || !x || !t) return fail(c, LPK_EINVAL, "bad gradient arguments");
    cudaSetDevice(c->device);
    const size_t bx = (sizeof(float) * (size_t)n * kF + 255) / 256 * 256;
    const size_t bt = (sizeof(float) * (size_t)n + 255) / 256 * 256;
    lpk_status s = ensure_scratch(c, bx + bt + 256);
    if (s) return s;
    float *d_x = (float *)c->d_scratch, *d_t = (float *)((char *)c->d_scratch + bx);
    float *d_loss = (float *)((char *)c->d_scratch + bx + bt);
    if ((s = upload(c, d_x, x, sizeof(float) * (size_t)n * kF)) || (s = upload(c, d_t, t, sizeof(float) * (size_t)n)))
        return s;
    cudaMemsetAsync(d_loss, 0, sizeof(float), c->stream);
    cudaMemsetAsync(m->d_g, 0, sizeof(float) * kParams, c->stream);
    if ((s = launch_grad(m, d_x, d_t, n, d_loss))) return s;
    float l = 0.0f;
    cudaError_t e = cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && grad)
        e = cudaMemcpyAsync(grad, m->d_g, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->d_g, 0, sizeof(float) * kParams, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp gradient read");
    if (loss) *loss = (double)l / (double)n;
    return LPK_OK;
}

lpk_status lpk_mlp_fit(lpk_mlp *m, const int32_t *tx, const lpk_kepler_orbit *orbits, int32_t n_tx, const double *rx,
                       int32_t n_rx, double epoch, double t0, double t1, int64_t n_train, int32_t steps, int32_t batch,
                       float lr, uint64_t seed, float *loss_curve) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    if (!rx || n_rx < 1) return fail(c, LPK_EINVAL, "fit needs at least one receiver");
    if (n_train < kRowsPerBlock || batch < kRowsPerBlock || batch > n_train || steps < 1 || !(lr > 0.0f) ||
        !(t1 > t0))
        return fail(c, LPK_EINVAL, "fit needs n_train >= batch >= 128, steps >= 1, lr > 0, t1 > t0");
    cudaSetDevice(c->device);
    lpk_status s = set_orbits(m, tx, orbits, n_tx);
    if (s) return s;
    float *d_x = nullptr, *d_y = nullptr, *d_curve = nullptr;
    int32_t *d_bad = nullptr;
    double *d_rx = nullptr;
    auto cleanup = [&]() {
        cudaStreamSynchronize(c->stream);
        for (void *p : {(void *)d_x, (void *)d_y, (void *)d_curve, (void *)d_bad, (void *)d_rx})
            if (p) cudaFree(p);
    };
    if (cudaMalloc(&d_x, sizeof(float) * (size_t)n_train * kF) != cudaSuccess ||
        cudaMalloc(&d_y, sizeof(float) * (size_t)n_train) != cudaSuccess ||
        cudaMalloc(&d_curve, sizeof(float) * (size_t)steps) != cudaSuccess ||
        cudaMalloc(&d_bad, sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&d_rx, sizeof(double) * 3 * (size_t)n_rx) != cudaSuccess) {
        cleanup();
        return fail(c, LPK_ENOMEM, "training set allocation failed");
    }
    cudaMemsetAsync(d_bad, 0, sizeof(int32_t), c->stream);
    cudaMemsetAsync(d_curve, 0, sizeof(float) * (size_t)steps, c->stream);
    if ((s = upload(c, d_rx, rx, sizeof(double) * 3 * (size_t)n_rx))) {
        cleanup();
        return s;
    }
    const unsigned g128 = (unsigned)((n_train + 127) / 128);
    k_mlp_dataset<<<g128, 128, 0, c->stream>>>(c->d_tx, m->d_scene_tx, m->d_el, n_tx, d_rx, n_rx, epoch, t0, t1,
                                                n_train, seed, d_x, d_y, d_bad);
    c->launches += 1;
    // normalisation from the first rows of the training set (host, double sums)
    const int64_t n_stat = std::min<int64_t>(n_train, (int64_t)1 << 21);
    std::vector<float> hx((size_t)n_stat * kF), hy((size_t)n_stat);
    int32_t bad = 0;
    cudaError_t e = cudaMemcpyAsync(hx.data(), d_x, sizeof(float) * hx.size(), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hy.data(), d_y, sizeof(float) * hy.size(), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(c, e, "training set");
    }
    if (bad) {
        cleanup();
        return fail(c, LPK_ENOCONV, "the converged solver did not converge on some training samples");
    }
    for (int k = 0; k <= kF; ++k) {
        double s1 = 0.0, s2 = 0.0;
        for (int64_t i = 0; i < n_stat; ++i) {
            const double v = k < kF ? hx[(size_t)i * kF + k] : hy[(size_t)i];
            s1 += v;
            s2 += v * v;
        }
        const double mean = s1 / (double)n_stat, var = std::max(0.0, s2 / (double)n_stat - mean * mean);
        const double sd = std::sqrt(var) > 1e-12 * std::max(1.0, std::fabs(mean)) ? std::sqrt(var) : 1.0;
        if (k < kF) {
            m->norm[k] = (float)mean;
            m->norm[kF + k] = (float)sd;
        } else {
            m->norm[2 * kF] = (float)mean;
            m->norm[2 * kF + 1] = (float)sd;
        }
    }
    if ((s = upload(c, m->d_norm, m->norm, sizeof m->norm))) {
        cleanup();
        return s;
    }
    k_mlp_normalize<<<g128, 128, 0, c->stream>>>(d_x, d_y, n_train, m->d_norm);
    c->launches += 1;
    // Adam with a cosine learning-rate decay over `steps` batches
    const int64_t span = n_train - batch + 1;
    for (int32_t k = 0; k < steps && !s; ++k) {
        const int64_t off = ((int64_t)k * batch) % span;
        s = launch_grad(m, d_x + off * kF, d_y + off, batch, d_curve + k);
        ++m->step;
        const float lrk = lr * 0.5f * (1.0f + cosf(3.14159265f * (float)k / (float)steps));
        const float bc1 = 1.0f - powf(0.9f, (float)m->step), bc2 = 1.0f - powf(0.999f, (float)m->step);
        k_mlp_adam<<<(kParams + 255) / 256, 256, 0, c->stream>>>(m->d_p, m->d_g, m->d_m, m->d_v, lrk, bc1, bc2);
        c->launches += 1;
    }
    if (!s && loss_curve) {
        e = cudaMemcpyAsync(loss_curve, d_curve, sizeof(float) * (size_t)steps, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_fail(c, e, "loss curve");
        for (int32_t k = 0; k < steps && !s; ++k) loss_curve[k] /= (float)batch;
    }
    if (!s && (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) s = cuda_fail(c, e, "mlp training");
    if (!s && (e = cudaGetLastError()) != cudaSuccess) s = cuda_fail(c, e, "mlp training");
    cleanup();
    return s;
}

lpk_status lpk_mlp_features(const lpk_mlp *m, int32_t tx, const double *rx, double epoch, const double *t_rel_utc,
                            int64_t n, float *features) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    if (!rx) return fail(c, LPK_EINVAL, "rx_ecef is NULL");
    if (tx < 0 || (size_t)tx >= m->k_of_tx.size() || m->k_of_tx[tx] < 0)
        return fail(c, LPK_EINVAL, "transmitter is not among the network's orbits");
    if (n < 0 || (n > 0 && (!t_rel_utc || !features))) return fail(c, LPK_EINVAL, "bad feature arguments");
    if (n == 0) return LPK_OK;
    cudaSetDevice(c->device);
    const size_t b_t = (sizeof(double) * (size_t)n + 255) / 256 * 256, b_r = 256;
    lpk_status s = ensure_scratch(c, b_t + b_r + sizeof(float) * (size_t)n * kF);
    if (s) return s;
    double *d_t = (double *)c->d_scratch, *d_r3 = (double *)((char *)c->d_scratch + b_t);
    float *d_x = (float *)((char *)c->d_scratch + b_t + b_r);
    if ((s = upload(c, d_t, t_rel_utc, sizeof(double) * (size_t)n)) || (s = upload(c, d_r3, rx, 3 * sizeof(double))))
        return s;
    k_elem_features<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(m->d_el, m->d_k_of_tx, nullptr, tx, d_r3,
                                                                        nullptr, epoch, d_t, n, nullptr, d_x, nullptr);
    c->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(features, d_x, sizeof(float) * (size_t)n * kF, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "mlp features");
}

lpk_status lpk_solve_converged(lpk_ctx *c, int32_t tx, const double *rx, double epoch, const double *t_rel_utc,
                               int64_t n, double tol_s, int32_t max_iter, int32_t scheme, int32_t start,
                               const lpk_mlp *m, double *t_emit, int32_t *iters, float *start_err) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    return solve_impl(c, nullptr, tx, rx, nullptr, 1, epoch, t_rel_utc, n, tol_s, max_iter, scheme, start, m, t_emit,
                      iters, start_err, nullptr);
}

lpk_status lpk_solve_converged_scene(lpk_ctx *c, const int32_t *tx, const int32_t *rx_idx, const double *rx_ecef,
                                     int32_t n_rx, double epoch, const double *t_rel_utc, int64_t n, double tol_s,
                                     int32_t max_iter, int32_t scheme, int32_t start, const lpk_mlp *m,
                                     double *t_emit, int32_t *iters, float *start_err, double *device_ms) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (n > 0 && (!tx || !rx_idx)) return fail(c, LPK_EINVAL, "tx or rx index array is NULL");
    return solve_impl(c, tx, 0, rx_ecef, rx_idx, n_rx, epoch, t_rel_utc, n, tol_s, max_iter, scheme, start, m, t_emit,
                      iters, start_err, device_ms);
}

}  // extern "C"
