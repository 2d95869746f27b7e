// lpk_mlp.cu — the learned warm start of the emission-time solve, and the
// converged solver it serves.
//
// The reference solves the emission time with two fixed-point iterations
// from t - 70 ms (src/channel/mod.rs:49-101). Where a converged solve is
// wanted (the delay truth, or a solver that iterates to a residual), each
// sample starts from one of:
//   LAG        the reference's initial guess, t - 70 ms;
//   GEOMETRIC  the range at the reception time, R(t) / c;
//   LEARNED    R(t) / c plus the light-time correction τ - R/c predicted by
//              a small MLP (8 -> 64 -> 64 -> 1, tanh) from the trajectory
//              state at t and the receiver position.
// Fixed-point or Newton iterations then finish the solve to the requested
// tolerance; a learned start that does not converge within the budget
// falls back to the LAG start, and the distance of every start from the
// converged delay is reported (the surrogate is judged, never trusted).
//
// The network is trained on this GPU from delays the converged solver
// itself produces, by the kernels below: inference and training's weight
// gradients run on the 5th-generation tensor cores (tcgen05.mma, BF16
// operands, FP32 accumulator in TMEM, 128-row tiles); training's forward
// and backward dH1 run as BF16 mma.sync tiles inside each warp's registers
// (16- to 64-wide products between layers); Adam updates FP32 master
// weights. Rounding points (BF16:
// inputs, W1, W2, the first hidden layer and the two pre-activation
// gradients; everything else FP32) are restated in oracle/mlp_ref.py.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "lpk_internal.h"
#include "lpk_split.cuh"

namespace lpk {
namespace {

constexpr int kF = 8;    // features
constexpr int kH = 64;   // hidden width
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kParams = kOffB3 + 1;  // 4801
constexpr int kLdX = 24;   // padded row strides (bf16 elements) of the shared tiles
constexpr int kLdH = 72;
constexpr int kRowsPerBlock = 128;  // 8 warps x 16 rows

struct __align__(16) MlpWeights {
    __nv_bfloat16 w1[kH][kLdX];   // W1 (out x in), inputs 8..15 zero
    __nv_bfloat16 w2[kH][kLdH];   // W2 (out x in)
    __nv_bfloat16 w2t[kH][kLdH];  // W2 transposed
    float b1[kH], b2[kH], w3[kH], b3;
};

// Weight gradients of one block step as one tcgen05 product, K = the
// step's 128 rows: A = [dZ2^T; dZ1^T] (128 x 128), B = [H1^T; X^T; 0]
// (80 x 128), so D = A B^T holds dW2 = dZ2^T H1 in rows 0-63 / columns 0-63
// and dW1 = dZ1^T X in rows 64-127 / columns 64-71 (the other blocks are
// not used). Both operands in the no-swizzle K-major core-matrix layout
// (element (row, k) at [k / 8][row][k % 8]).
constexpr int kGradN = 80;
constexpr uint32_t kGradCols = 128;  // TMEM columns (a power of two >= kGradN)
constexpr uint32_t kGradIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kGradN >> 3) << 17) |
                                ((uint32_t)(kRowsPerBlock >> 4) << 24);

struct __align__(16) MlpTiles {  // one block step of 128 rows (training)
    __nv_bfloat16 ga[kRowsPerBlock / 8][2 * kH][8];
    __nv_bfloat16 gb[kRowsPerBlock / 8][kGradN][8];
    float db1[kH], db2[kH], dw3[kH], db3, loss;
    unsigned long long bar;
    uint32_t tmem;
};
// At most four gradient CTAs (their weights and tiles) fit on an SM's
// 228 KB, so their TMEM (4 x 128 columns) never exceeds the SM's 512.
static_assert(5 * (sizeof(MlpWeights) + sizeof(MlpTiles)) > 228 * 1024 && 4 * kGradCols <= 512,
              "TMEM residency bound");

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
    for (int i = threadIdx.x; i < kH * kLdX; i += blockDim.x) {
        const int o = i / kLdX, k = i % kLdX;
        S.w1[o][k] = __float2bfloat16_rn(k < kF ? p[kOffW1 + o * kF + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int o = i / kH, k = i % kH;
        const __nv_bfloat16 w = __float2bfloat16_rn(p[kOffW2 + i]);
        S.w2[o][k] = w;
        S.w2t[k][o] = w;
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        S.b1[i] = p[kOffB1 + i];
        S.b2[i] = p[kOffB2 + i];
        S.w3[i] = p[kOffW3 + i];
    }
    if (threadIdx.x == 0) S.b3 = p[kOffB3];
}

// Forward pass of one warp's 16 rows. xg / xg8: this thread's inputs
// (columns 2·tig, 2·tig+1) of rows g and g+8. Leaves the tanh outputs of
// both hidden layers in fragment layout (h[j][e]: n-tile j, element e) and
// returns y for rows g (y[0]) and g+8 (y[1]) in every thread of the group.
struct WarpAct {
    float h1[8][4], h2[8][4];
    uint32_t a2[4][4];  // BF16 A fragments of h1 (the second layer's input)
};

__device__ __forceinline__ void warp_forward(const MlpWeights &S, float2 xg, float2 xg8, WarpAct &A, float y[2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    const uint32_t ax[4] = {pack2(xg.x, xg.y), pack2(xg8.x, xg8.y), 0u, 0u};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {S.b1[8 * j + 2 * tig], S.b1[8 * j + 2 * tig + 1], S.b1[8 * j + 2 * tig],
                        S.b1[8 * j + 2 * tig + 1]};
        mma16816(acc, ax, ld2(&S.w1[8 * j + g][2 * tig]), 0u);
#pragma unroll
        for (int e = 0; e < 4; ++e) A.h1[j][e] = tanhf(acc[e]);
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        A.a2[kk][0] = pack2(A.h1[2 * kk][0], A.h1[2 * kk][1]);
        A.a2[kk][1] = pack2(A.h1[2 * kk][2], A.h1[2 * kk][3]);
        A.a2[kk][2] = pack2(A.h1[2 * kk + 1][0], A.h1[2 * kk + 1][1]);
        A.a2[kk][3] = pack2(A.h1[2 * kk + 1][2], A.h1[2 * kk + 1][3]);
    }
    float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc[4] = {S.b2[8 * j + 2 * tig], S.b2[8 * j + 2 * tig + 1], S.b2[8 * j + 2 * tig],
                        S.b2[8 * j + 2 * tig + 1]};
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            mma16816(acc, A.a2[kk], ld2(&S.w2[8 * j + g][16 * kk + 2 * tig]),
                     ld2(&S.w2[8 * j + g][16 * kk + 8 + 2 * tig]));
#pragma unroll
        for (int e = 0; e < 4; ++e) A.h2[j][e] = tanhf(acc[e]);
        const float wa = S.w3[8 * j + 2 * tig], wb = S.w3[8 * j + 2 * tig + 1];
        s0 = fmaf(A.h2[j][0], wa, fmaf(A.h2[j][1], wb, s0));
        s1 = fmaf(A.h2[j][2], wa, fmaf(A.h2[j][3], wb, s1));
    }
    s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
    s0 += __shfl_xor_sync(0xffffffffu, s0, 2);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
    s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
    y[0] = s0 + S.b3;
    y[1] = s1 + S.b3;
}

__device__ __forceinline__ float2 load_x2(const float *__restrict__ x, int64_t row, int64_t n, int tig) {
    if (row >= n) return make_float2(0.0f, 0.0f);
    return make_float2(x[row * kF + 2 * tig], x[row * kF + 2 * tig + 1]);
}

constexpr int kTcRows = 128;          // rows per tile = the MMA's M
constexpr uint32_t kTcCols = 64;      // TMEM columns: one 128 x 64 FP32 accumulator, reused by both layers
// kind::f16 instruction descriptor: FP32 accumulator (bits 4-5 = 1), BF16 A
// (7-9 = 1) and B (10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kH >> 3) << 17) |
                              ((uint32_t)(kTcRows >> 4) << 24);
constexpr int kTcSpin = 1 << 20;      // mbarrier polls before a wait gives up

struct __align__(1024) TcSmem {
    __nv_bfloat16 a1[2][kTcRows][8];  // x tile, K padded to 16: column groups 0-7 and 8-15 (zero)
    __nv_bfloat16 a2[kH / 8][kTcRows][8];  // first hidden layer, 8 column groups
    __nv_bfloat16 b1[2][kH][8];       // W1 (out x in), K padded to 16
    __nv_bfloat16 b2[kH / 8][kH][8];  // W2 (out x in)
    float bias1[kH], bias2[kH], w3[kH];
    float b3;
    unsigned long long bar;
    uint32_t tmem;
};
// At most 7 CTAs of 29 KB or more fit on an SM (228 KB), so their TMEM
// demand (7 x 64 columns) stays within the SM's 512 and tcgen05.alloc never
// waits on another CTA.
static_assert(sizeof(TcSmem) >= 29 * 1024 && 7 * kTcCols <= 512, "TMEM residency bound");

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

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t phase) {
    for (int it = 0; it < kTcSpin; ++it) {
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

// This warp's 32 accumulator rows, 16 FP32 columns from taddr's column.
__device__ __forceinline__ void tc_load16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
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

// Gradient of L = (1/N) Σ (y - t)² over n rows (N = n_total) into grad
// (FP32, accumulated with atomics) and Σ (y - t)² into loss. Each block
// step takes 128 rows: 8 warps run forward and backward on 16 rows each in
// registers, stage the BF16 operands of the weight gradients in shared
// memory, and the weight gradients are tensor-core tiles summed over the
// 128 rows (dW2: 32 tiles of 16x8, four per warp; dW1: 4 tiles).
__global__ void __launch_bounds__(256) k_mlp_grad(const float *__restrict__ p, const float *__restrict__ x,
                                                  const float *__restrict__ t, int64_t n, float two_over_n,
                                                  float *__restrict__ grad, float *__restrict__ loss,
                                                  int *__restrict__ err) {
    __shared__ MlpWeights S;
    extern __shared__ __align__(16) unsigned char tiles_raw[];
    MlpTiles &T = *reinterpret_cast<MlpTiles *>(tiles_raw);
    stage_weights(p, S);
    for (int i = threadIdx.x; i < (kRowsPerBlock / 8) * (kGradN - kH - kF) * 8; i += blockDim.x) {
        const int kg = i / ((kGradN - kH - kF) * 8), rest = i % ((kGradN - kH - kF) * 8);
        T.gb[kg][kH + kF + rest / 8][rest % 8] = __float2bfloat16_rn(0.0f);  // B rows 72-79 stay zero
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) T.db1[i] = T.db2[i] = T.dw3[i] = 0.0f;
    if (threadIdx.x == 0) {
        T.db3 = T.loss = 0.0f;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&T.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, tig = lane & 3;
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&T.tmem)),
                     "r"(kGradCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = T.tmem, bar = smem_u32(&T.bar);
    uint32_t phase = 0;
    bool ok = true;
    int64_t steps = 0;
    for (int64_t r0 = (int64_t)blockIdx.x * kRowsPerBlock; r0 < n && ok;
         r0 += (int64_t)gridDim.x * kRowsPerBlock, ++steps) {
        const int64_t ra = r0 + 16 * w + g, rb = ra + 8;
        const float2 xa = load_x2(x, ra, n, tig), xb = load_x2(x, rb, n, tig);
        WarpAct A;
        float y[2];
        warp_forward(S, xa, xb, A, y);
        const float ea = ra < n ? y[0] - t[ra] : 0.0f, eb = rb < n ? y[1] - t[rb] : 0.0f;
        const float dya = ea * two_over_n, dyb = eb * two_over_n;
        // loss and db3: one count per row (tig == 0)
        const float l = rows_sum(tig == 0 ? ea * ea : 0.0f, tig == 0 ? eb * eb : 0.0f);
        const float d3 = rows_sum(tig == 0 ? dya : 0.0f, tig == 0 ? dyb : 0.0f);
        if (lane == 0) {
            atomicAdd(&T.loss, l);
            atomicAdd(&T.db3, d3);
        }
        // dZ2 = dy w3 (1 - h2²); dw3 += dy h2; db2 += dZ2
        float dz2[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float dy = e < 2 ? dya : dyb;
                const float wv = S.w3[8 * j + 2 * tig + (e & 1)];
                dz2[j][e] = dy * wv * (1.0f - A.h2[j][e] * A.h2[j][e]);
            }
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float s3 = rows_sum(dya * A.h2[j][e], dyb * A.h2[j][e + 2]);
                const float s2 = rows_sum(dz2[j][e], dz2[j][e + 2]);
                if (g == 0) {
                    atomicAdd(&T.dw3[8 * j + 2 * tig + e], s3);
                    atomicAdd(&T.db2[8 * j + 2 * tig + e], s2);
                }
            }
        }
        uint32_t adz2[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            adz2[kk][0] = pack2(dz2[2 * kk][0], dz2[2 * kk][1]);
            adz2[kk][1] = pack2(dz2[2 * kk][2], dz2[2 * kk][3]);
            adz2[kk][2] = pack2(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
            adz2[kk][3] = pack2(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
        }
        // dH1 = dZ2 W2 (tensor cores), dZ1 = dH1 (1 - h1²); db1 += dZ1
        const int ra_s = 16 * w + g, rb_s = ra_s + 8;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                mma16816(acc, adz2[kk], ld2(&S.w2t[8 * j + g][16 * kk + 2 * tig]),
                         ld2(&S.w2t[8 * j + g][16 * kk + 8 + 2 * tig]));
            float dz1[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) dz1[e] = acc[e] * (1.0f - A.h1[j][e] * A.h1[j][e]);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float s1 = rows_sum(dz1[e], dz1[e + 2]);
                if (g == 0) atomicAdd(&T.db1[8 * j + 2 * tig + e], s1);
            }
            // operands of the weight gradients, transposed into the K-major
            // tiles (K = the step's row): rows ra_s / rb_s, columns c, c + 1
            const int c = 8 * j + 2 * tig;
            T.ga[ra_s >> 3][c][ra_s & 7] = __float2bfloat16_rn(dz2[j][0]);
            T.ga[ra_s >> 3][c + 1][ra_s & 7] = __float2bfloat16_rn(dz2[j][1]);
            T.ga[rb_s >> 3][c][rb_s & 7] = __float2bfloat16_rn(dz2[j][2]);
            T.ga[rb_s >> 3][c + 1][rb_s & 7] = __float2bfloat16_rn(dz2[j][3]);
            T.ga[ra_s >> 3][kH + c][ra_s & 7] = __float2bfloat16_rn(dz1[0]);
            T.ga[ra_s >> 3][kH + c + 1][ra_s & 7] = __float2bfloat16_rn(dz1[1]);
            T.ga[rb_s >> 3][kH + c][rb_s & 7] = __float2bfloat16_rn(dz1[2]);
            T.ga[rb_s >> 3][kH + c + 1][rb_s & 7] = __float2bfloat16_rn(dz1[3]);
            T.gb[ra_s >> 3][c][ra_s & 7] = __float2bfloat16_rn(A.h1[j][0]);
            T.gb[ra_s >> 3][c + 1][ra_s & 7] = __float2bfloat16_rn(A.h1[j][1]);
            T.gb[rb_s >> 3][c][rb_s & 7] = __float2bfloat16_rn(A.h1[j][2]);
            T.gb[rb_s >> 3][c + 1][rb_s & 7] = __float2bfloat16_rn(A.h1[j][3]);
        }
        T.gb[ra_s >> 3][kH + 2 * tig][ra_s & 7] = __float2bfloat16_rn(xa.x);
        T.gb[ra_s >> 3][kH + 2 * tig + 1][ra_s & 7] = __float2bfloat16_rn(xa.y);
        T.gb[rb_s >> 3][kH + 2 * tig][rb_s & 7] = __float2bfloat16_rn(xb.x);
        T.gb[rb_s >> 3][kH + 2 * tig + 1][rb_s & 7] = __float2bfloat16_rn(xb.y);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> the MMA's reads
        tc_fence_before();
        __syncthreads();
        // weight gradients over the block's 128 rows, accumulated in TMEM
        // over the block's steps: eight K = 16 MMAs of M = 128, N = 80
        if (threadIdx.x == 0) {
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < kRowsPerBlock / 16; ++kk)
                tc_mma(tmem, tc_desc(smem_u32(&T.ga[2 * kk][0][0]), 2 * kH * 16, 128),
                       tc_desc(smem_u32(&T.gb[2 * kk][0][0]), kGradN * 16, 128),
                       (steps > 0 || kk > 0) ? 1u : 0u, kGradIdesc);
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase));  // the tiles are rewritten by the next step
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();  // the next step overwrites the tiles
    }
    if (!ok && threadIdx.x == 0 && err) atomicOr(err, 1);
    // Warps w and w + 4 share TMEM lane quarter w % 4 (accumulator rows
    // 32 (w % 4) ..): quarters 0-1 hold dW2, each warp of the pair reading
    // 32 of its 64 columns; quarters 2-3 hold dW1 in columns 64-71.
    const int q = w & 3, half = w >> 2;
    if (ok && steps > 0 && (q < 2 || half == 0)) {
        const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16);
        const int m = 32 * q + lane;
        float v[16];
        if (q < 2) {
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const int c0 = 32 * half + 16 * part;
                tc_load16(taddr + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(&grad[kOffW2 + m * kH + c0 + i], v[i]);
            }
        } else {
            tc_load16(taddr + (uint32_t)kH, v);
#pragma unroll
            for (int f = 0; f < kF; ++f) atomicAdd(&grad[kOffW1 + (m - kH) * kF + f], v[f]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGradCols) : "memory");
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        atomicAdd(&grad[kOffB1 + i], T.db1[i]);
        atomicAdd(&grad[kOffB2 + i], T.db2[i]);
        atomicAdd(&grad[kOffW3 + i], T.dw3[i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grad[kOffB3], T.db3);
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

// ------------------------------------------------------------------ solver
// Trajectory state at the reception time tu (no light time): features of
// the network and the geometric range R. Position and velocity come from
// the lerp table on its natural segment, without rounding epoch + t.
__device__ __forceinline__ void solve_features(const DevTx &tx, double tu, double de, double ox, double oy,
                                               double oz, float f[kF], double &R) {
    bool cl;
    const int64_t lo = seg_unrounded(tx, tu, de, cl);
    double px, py, pz, vx = 0.0, vy = 0.0, vz = 0.0;
    pos_unrounded(tx, tu, de, lo, px, py, pz);
    if (tx.traj_kind != 0) {
        const double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
        vx = (b.x - a.x) / tx.dt;
        vy = (b.y - a.y) / tx.dt;
        vz = (b.z - a.z) / tx.dt;
    }
    const double dx = px - ox, dy = py - oy, dz = pz - oz;
    R = sqrt(dx * dx + dy * dy + dz * dz);
    const double inv = R > 0.0 ? 1.0 / R : 0.0, ic = 1.0 / kSpeedOfLight;
    const double ux = dx * inv, uy = dy * inv, uz = dz * inv;
    f[0] = (float)ux;
    f[1] = (float)uy;
    f[2] = (float)uz;
    f[3] = (float)(R * ic);
    f[4] = (float)((vx * ux + vy * uy + vz * uz) * ic);
    f[5] = (float)(vx * ic);
    f[6] = (float)(vy * ic);
    f[7] = (float)(kEarthRate * (px * oy - py * ox) * inv * ic);  // Sagnac rate of the line of sight
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
// GEOMETRIC / LEARNED start does not converge.
__global__ void __launch_bounds__(128)
k_solve_converged(const DevTx *__restrict__ txs, int32_t tx_idx, double ox, double oy, double oz, double epoch,
                  const double *__restrict__ tu, int64_t n, double tol, int32_t max_iter, int32_t scheme,
                  int32_t start, const float *__restrict__ pred, float tmean, float tstd, double *__restrict__ temit,
                  int32_t *__restrict__ iters, float *__restrict__ start_err) {
    __shared__ DevTx stx;
    if (threadIdx.x == 0) stx = txs[tx_idx];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double de = stx.traj_kind != 0 ? epoch - stx.t0 : 0.0;
    const double t = tu[i];
    double tau0 = kLagStart;
    if (start != 0) {
        float f[kF];
        double R;
        solve_features(stx, t, de, ox, oy, oz, f, R);
        tau0 = R / kSpeedOfLight;
        if (start == 2) tau0 += (double)fmaf(pred[i], tstd, tmean) * 1e-6;  // correction in µs
    }
    double tau;
    int it = converge(stx, t, de, ox, oy, oz, tol, max_iter, scheme, tau0, tau);
    if (it < 0 && start != 0) {
        int it2 = converge(stx, t, de, ox, oy, oz, tol, max_iter, scheme, kLagStart, tau);
        it = it2 < 0 ? -1 : max_iter + it2;
    }
    temit[i] = t - tau;
    iters[i] = it;
    if (start_err) start_err[i] = (float)fabs(tau0 - tau);
}

// Normalised features of n samples (the learned start's input).
__global__ void __launch_bounds__(128)
k_solve_features(const DevTx *__restrict__ txs, int32_t tx_idx, double ox, double oy, double oz, double epoch,
                 const double *__restrict__ tu, int64_t n, const float *__restrict__ norm, float *__restrict__ x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevTx &tx = txs[tx_idx];
    const double de = tx.traj_kind != 0 ? epoch - tx.t0 : 0.0;
    float f[kF];
    double R;
    solve_features(tx, tu[i], de, ox, oy, oz, f, R);
#pragma unroll
    for (int k = 0; k < kF; ++k) x[i * kF + k] = norm ? (f[k] - norm[k]) / norm[kF + k] : f[k];
}

// Training set: reception times uniform in [t0, t1) (Philox counter i, tag
// "MLPT"), raw features, and the light-time correction τ - R/c (µs) of the
// converged Newton solve from the geometric start.
__global__ void __launch_bounds__(128)
k_mlp_dataset(const DevTx *__restrict__ txs, int32_t tx_idx, double ox, double oy, double oz, double epoch,
              double t0, double t1, int64_t n, uint64_t seed, float *__restrict__ x, float *__restrict__ y,
              int32_t *__restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevTx &tx = txs[tx_idx];
    const uint4 r = philox4x32_10(make_uint4((uint32_t)(uint64_t)i, (uint32_t)((uint64_t)i >> 32), 0x4D4C5054u, 0u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double u = (double)(((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11)) * 0x1.0p-53;
    const double t = t0 + (t1 - t0) * u;
    const double de = tx.traj_kind != 0 ? epoch - tx.t0 : 0.0;
    float f[kF];
    double R, tau;
    solve_features(tx, t, de, ox, oy, oz, f, R);
    const int it = converge(tx, t, de, ox, oy, oz, 1e-16, 20, 1, R / kSpeedOfLight, tau);
    if (it < 0) atomicAdd(bad, 1);
#pragma unroll
    for (int k = 0; k < kF; ++k) x[i * kF + k] = f[k];
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
// tiles of 128 rows: the tile's inputs and hidden layer are staged in shared
// memory in the no-swizzle K-major core-matrix layout that tcgen05.mma reads
// (8 rows x 16 bytes per core matrix; next 8-row group +128 B, next 8
// K-elements +rows*16 B), one thread issues the MMAs (M = 128, N = 64,
// K = 16 per instruction, BF16 operands, FP32 accumulator in TMEM), commits
// them to an mbarrier, and each warp reads its 32 rows of the accumulator
// back with tcgen05.ld for the tanh epilogue. Rounding points are those of
// the mma.sync kernels (BF16 x, W1, W2 and first hidden layer; FP32
// accumulation and everything else), so the CPU restatement covers both;
// only the FP32 summation order differs (bias added after the products).
// y = MLP(x) for n rows of normalised features; err (may be NULL) gets 1 if
// an MMA completion wait gave up (the outputs are then incomplete).
__global__ void __launch_bounds__(128, 1) k_mlp_forward_tc(const float *__restrict__ p, const float *__restrict__ x,
                                                           int64_t n, float *__restrict__ y, int *__restrict__ err) {
    __shared__ TcSmem S;
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights in the core-matrix layout (W1's K padded with zeros), biases,
    // and the zero half of the input tile
    for (int i = tid; i < 2 * kH * 8; i += blockDim.x) {
        const int g = i / (kH * 8), o = (i / 8) % kH, c = i % 8, k = 8 * g + c;
        S.b1[g][o][c] = __float2bfloat16_rn(k < kF ? p[kOffW1 + o * kF + k] : 0.0f);
    }
    for (int i = tid; i < kH * kH; i += blockDim.x) {
        const int o = i / kH, k = i % kH;
        S.b2[k / 8][o][k % 8] = __float2bfloat16_rn(p[kOffW2 + i]);
    }
    for (int i = tid; i < kH; i += blockDim.x) {
        S.bias1[i] = p[kOffB1 + i];
        S.bias2[i] = p[kOffB2 + i];
        S.w3[i] = p[kOffW3 + i];
    }
    for (int i = tid; i < kTcRows * 8; i += blockDim.x) S.a1[1][i / 8][i % 8] = __float2bfloat16_rn(0.0f);
    if (tid == 0) {
        S.b3 = p[kOffB3];
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
        // inputs of this thread's row, BF16, into column group 0 of the tile
        {
            float v[kF];
#pragma unroll
            for (int k = 0; k < kF; ++k) v[k] = row < n ? x[row * kF + k] : 0.0f;
            uint4 pk;
            pk.x = pack2(v[0], v[1]);
            pk.y = pack2(v[2], v[3]);
            pk.z = pack2(v[4], v[5]);
            pk.w = pack2(v[6], v[7]);
            *reinterpret_cast<uint4 *>(&S.a1[0][tid][0]) = pk;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> the MMA's reads
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            tc_mma(tmem, d_a1, d_b1, 0u, kTcIdesc);  // layer 1: one K = 16 step
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        float h[kH];
        tc_load_row(trow, h);
#pragma unroll
        for (int g = 0; g < kH / 8; ++g) {  // tanh, BF16, into the second layer's A tile
            uint4 pk;
            pk.x = pack2(tanhf(h[8 * g + 0] + S.bias1[8 * g + 0]), tanhf(h[8 * g + 1] + S.bias1[8 * g + 1]));
            pk.y = pack2(tanhf(h[8 * g + 2] + S.bias1[8 * g + 2]), tanhf(h[8 * g + 3] + S.bias1[8 * g + 3]));
            pk.z = pack2(tanhf(h[8 * g + 4] + S.bias1[8 * g + 4]), tanhf(h[8 * g + 5] + S.bias1[8 * g + 5]));
            pk.w = pack2(tanhf(h[8 * g + 6] + S.bias1[8 * g + 6]), tanhf(h[8 * g + 7] + S.bias1[8 * g + 7]));
            *reinterpret_cast<uint4 *>(&S.a2[g][tid][0]) = pk;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();  // every warp has read the layer-1 accumulator and written its rows
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < kH / 16; ++kk)  // layer 2: four K = 16 steps
                tc_mma(tmem, tc_desc(smem_u32(&S.a2[2 * kk][0][0]), kTcRows * 16, 128),
                       tc_desc(smem_u32(&S.b2[2 * kk][0][0]), kH * 16, 128), kk > 0 ? 1u : 0u, kTcIdesc);
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        tc_load_row(trow, h);
        float s = 0.0f;
#pragma unroll
        for (int c = 0; c < kH; ++c) s = fmaf(tanhf(h[c] + S.bias2[c]), S.w3[c], s);
        if (row < n) y[row] = s + S.b3;
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
                               cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (e != cudaSuccess || n <= 0) return e;
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    // five CTAs per SM: what the kernel's 96 registers allow (and 5 x 64 TMEM columns fit)
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 5 * (int64_t)sms));
    k_mlp_forward_tc<<<grid, 128, 0, st>>>(d_p, d_x, n, d_y, d_err);
    return cudaGetLastError();
}

}  // namespace
}  // namespace lpk

using namespace lpk;

struct lpk_mlp {
    lpk_ctx *ctx = nullptr;
    float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr, *d_norm = nullptr;
    int *d_err = nullptr;  // set by the gradient kernel when a tensor-core completion wait gives up
    float norm[2 * kF + 2];  // feature means, feature stds, target mean, target std (µs)
    int64_t step = 0;
};

namespace {

size_t grad_smem() { return sizeof(MlpTiles); }

lpk_status upload(lpk_ctx *c, void *dst, const void *src, size_t bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "upload");
}

lpk_status launch_grad(lpk_mlp *m, const float *d_x, const float *d_t, int64_t n, float *d_loss) {
    lpk_ctx *c = m->ctx;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem());
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp gradient shared memory");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int64_t steps = (n + kRowsPerBlock - 1) / kRowsPerBlock;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(steps, 2 * sms));
    k_mlp_grad<<<grid, 256, grad_smem(), c->stream>>>(m->d_p, d_x, d_t, n, 2.0f / (float)n, m->d_g, d_loss,
                                                      m->d_err);
    e = cudaGetLastError();
    c->launches += 1;
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "mlp gradient kernel");
}

lpk_status txo_check(lpk_ctx *c, int32_t tx, const double *rx) {
    if (tx < 0 || tx >= c->n_tx) return fail(c, LPK_EINVAL, "transmitter index out of range of the uploaded scene");
    if (!rx) return fail(c, LPK_EINVAL, "rx_ecef is NULL");
    return LPK_OK;
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
        cudaError_t e = cudaMalloc((void **)bufs[k], sizeof(float) * (k == 4 ? 2 * kF + 2 : kParams));
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
    const double a1 = std::sqrt(6.0 / (kF + kH)), a2 = std::sqrt(6.0 / (kH + kH)), a3 = std::sqrt(6.0 / (kH + 1));
    for (int i = 0; i < kH * kF; ++i) p[kOffW1 + i] = (float)(a1 * uni());
    for (int i = 0; i < kH * kH; ++i) p[kOffW2 + i] = (float)(a2 * uni());
    for (int i = 0; i < kH; ++i) p[kOffW3 + i] = (float)(a3 * uni());
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
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "mlp gradient read");
    if (herr) return fail(c, LPK_ETIMEDOUT, "mlp gradient: a tensor-core completion wait gave up");
    if (loss) *loss = (double)l / (double)n;
    return LPK_OK;
}

lpk_status lpk_mlp_fit(lpk_mlp *m, int32_t tx, const double *rx, double epoch, double t0, double t1,
                       int64_t n_train, int32_t steps, int32_t batch, float lr, uint64_t seed, float *loss_curve) {
    if (!m) return fail(nullptr, LPK_EINVAL, "mlp is NULL");
    lpk_ctx *c = m->ctx;
    lpk_status s = txo_check(c, tx, rx);
    if (s) return s;
    if (n_train < kRowsPerBlock || batch < kRowsPerBlock || batch > n_train || steps < 1 || !(lr > 0.0f) ||
        !(t1 > t0))
        return fail(c, LPK_EINVAL, "fit needs n_train >= batch >= 128, steps >= 1, lr > 0, t1 > t0");
    cudaSetDevice(c->device);
    float *d_x = nullptr, *d_y = nullptr, *d_curve = nullptr;
    int32_t *d_bad = nullptr;
    auto cleanup = [&]() {
        cudaStreamSynchronize(c->stream);
        for (void *p : {(void *)d_x, (void *)d_y, (void *)d_curve, (void *)d_bad})
            if (p) cudaFree(p);
    };
    if (cudaMalloc(&d_x, sizeof(float) * (size_t)n_train * kF) != cudaSuccess ||
        cudaMalloc(&d_y, sizeof(float) * (size_t)n_train) != cudaSuccess ||
        cudaMalloc(&d_curve, sizeof(float) * (size_t)steps) != cudaSuccess ||
        cudaMalloc(&d_bad, sizeof(int32_t)) != cudaSuccess) {
        cleanup();
        return fail(c, LPK_ENOMEM, "training set allocation failed");
    }
    cudaMemsetAsync(d_bad, 0, sizeof(int32_t), c->stream);
    cudaMemsetAsync(d_curve, 0, sizeof(float) * (size_t)steps, c->stream);
    const unsigned g128 = (unsigned)((n_train + 127) / 128);
    k_mlp_dataset<<<g128, 128, 0, c->stream>>>(c->d_tx, tx, rx[0], rx[1], rx[2], epoch, t0, t1, n_train, seed, d_x,
                                                d_y, d_bad);
    c->launches += 1;
    // normalisation from the training set (host, double sums)
    std::vector<float> hx((size_t)n_train * kF), hy((size_t)n_train);
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
        for (int64_t i = 0; i < n_train; ++i) {
            const double v = k < kF ? hx[(size_t)i * kF + k] : hy[(size_t)i];
            s1 += v;
            s2 += v * v;
        }
        const double mean = s1 / (double)n_train, var = std::max(0.0, s2 / (double)n_train - mean * mean);
        const double sd = std::sqrt(var) > 1e-12 ? std::sqrt(var) : 1.0;
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
    int herr = 0;
    if (!s) {
        e = cudaMemcpyAsync(&herr, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) s = cuda_fail(c, e, "mlp training");
    }
    if (!s && (e = cudaGetLastError()) != cudaSuccess) s = cuda_fail(c, e, "mlp training");
    cleanup();
    if (!s && herr) s = fail(c, LPK_ETIMEDOUT, "mlp training: a tensor-core completion wait gave up");
    return s;
}

lpk_status lpk_solve_converged(lpk_ctx *c, int32_t tx, const double *rx, double epoch, const double *t_rel_utc,
                               int64_t n, double tol_s, int32_t max_iter, int32_t scheme, int32_t start,
                               const lpk_mlp *m, double *t_emit, int32_t *iters, float *start_err) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    lpk_status s = txo_check(c, tx, rx);
    if (s) return s;
    if (n < 0 || (n > 0 && (!t_rel_utc || !t_emit || !iters))) return fail(c, LPK_EINVAL, "bad solve arguments");
    if (scheme != LPK_ITER_FIXED_POINT && scheme != LPK_ITER_NEWTON) return fail(c, LPK_EINVAL, "unknown scheme");
    if (start != LPK_START_LAG && start != LPK_START_GEOMETRIC && start != LPK_START_LEARNED)
        return fail(c, LPK_EINVAL, "unknown start");
    if (start == LPK_START_LEARNED && (!m || m->ctx != c))
        return fail(c, LPK_EINVAL, "learned start needs an mlp of this context");
    if (!(tol_s >= 0.0) || max_iter < 1) return fail(c, LPK_EINVAL, "tol must be >= 0 and max_iter >= 1");
    if (n == 0) return LPK_OK;
    cudaSetDevice(c->device);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_t = al(sizeof(double) * (size_t)n), b_o = al(sizeof(double) * (size_t)n),
                 b_i = al(sizeof(int32_t) * (size_t)n), b_e = al(sizeof(float) * (size_t)n),
                 b_x = start == LPK_START_LEARNED ? al(sizeof(float) * (size_t)n * kF) : 0,
                 b_p = start == LPK_START_LEARNED ? al(sizeof(float) * (size_t)n) : 0, b_r = al(sizeof(int));
    if ((s = ensure_scratch(c, b_t + b_o + b_i + b_e + b_x + b_p + b_r))) return s;
    char *base = (char *)c->d_scratch;
    double *d_t = (double *)base, *d_o = (double *)(base + b_t);
    int32_t *d_i = (int32_t *)(base + b_t + b_o);
    float *d_e = (float *)(base + b_t + b_o + b_i), *d_x = (float *)(base + b_t + b_o + b_i + b_e);
    float *d_p = (float *)(base + b_t + b_o + b_i + b_e + b_x);
    int *d_err = (int *)(base + b_t + b_o + b_i + b_e + b_x + b_p);
    if ((s = upload(c, d_t, t_rel_utc, sizeof(double) * (size_t)n))) return s;
    const unsigned grid = (unsigned)((n + 127) / 128);
    if (start == LPK_START_LEARNED) {
        k_solve_features<<<grid, 128, 0, c->stream>>>(c->d_tx, tx, rx[0], rx[1], rx[2], epoch, d_t, n, m->d_norm, d_x);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        cudaError_t fe = launch_mlp_forward(m->d_p, d_x, n, d_p, d_err, sms, c->stream);
        if (fe != cudaSuccess) return cuda_fail(c, fe, "mlp forward");
        c->launches += 2;
    }
    k_solve_converged<<<grid, 128, 0, c->stream>>>(c->d_tx, tx, rx[0], rx[1], rx[2], epoch, d_t, n, tol_s, max_iter,
                                                   scheme, start, d_p, m ? m->norm[2 * kF] : 0.0f,
                                                   m ? m->norm[2 * kF + 1] : 1.0f, d_o, d_i, start_err ? d_e : nullptr);
    c->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(t_emit, d_o, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(iters, d_i, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && start_err)
        e = cudaMemcpyAsync(start_err, d_e, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    int herr = 0;
    if (e == cudaSuccess && start == LPK_START_LEARNED)
        e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "converged solve");
    return herr ? fail(c, LPK_ETIMEDOUT, "learned start: a tensor-core completion wait gave up") : LPK_OK;
}

lpk_status lpk_solve_features(lpk_ctx *c, int32_t tx, const double *rx, double epoch, const double *t_rel_utc,
                              int64_t n, float *features) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    lpk_status s = txo_check(c, tx, rx);
    if (s) return s;
    if (n < 0 || (n > 0 && (!t_rel_utc || !features))) return fail(c, LPK_EINVAL, "bad feature arguments");
    if (n == 0) return LPK_OK;
    cudaSetDevice(c->device);
    const size_t b_t = (sizeof(double) * (size_t)n + 255) / 256 * 256;
    if ((s = ensure_scratch(c, b_t + sizeof(float) * (size_t)n * kF))) return s;
    double *d_t = (double *)c->d_scratch;
    float *d_x = (float *)((char *)c->d_scratch + b_t);
    if ((s = upload(c, d_t, t_rel_utc, sizeof(double) * (size_t)n))) return s;
    k_solve_features<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(c->d_tx, tx, rx[0], rx[1], rx[2], epoch, d_t,
                                                                         n, nullptr, d_x);
    c->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(features, d_x, sizeof(float) * (size_t)n * kF, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "solve features");
}

}  // extern "C"
