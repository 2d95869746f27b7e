// lpk_walk.cuh — the device clock walk, shared by the single-band and
// batched paths so that both produce the same bits.
//
// The walk ε(k) = Σ_{j<=k} σ z_j (white frequency noise integrated at the
// master rate, ClockStream::advance_to, src/clock/mod.rs:299-307) is
// defined through a fixed summation tree over master indices, so nothing
// depends on how a band is chunked or which call computes which part:
//  * scan blocks of kWalkBlock master samples: P_b(k), the in-block
//    inclusive prefix in one fixed parallel order, and the block total t_b;
//  * carry(b) = Σ_{b'<b} t_b', summed in a fixed three-level order: 32-block
//    chunks (warp scan), 32-chunk groups (warp scan of the chunk sums), and
//    the group sums added one after another from group 0;
//  * ε(k) = carry(b) ⊕ P_b(k).
#pragma once

#include "lpk_device.cuh"

namespace lpk {

constexpr int64_t kWalkBlock = 4096;  // master samples per scan block
constexpr int kWalkThreads = 256;
#ifndef LPK_WALK_MINB
#define LPK_WALK_MINB 4  // scan blocks per SM (64 registers)
#endif
constexpr int kWalkPer = (int)(kWalkBlock / kWalkThreads);  // 16
constexpr int64_t kGroupBlocks = 1024;                      // scan blocks per carry group
constexpr int kGroupThreads = (int)kGroupBlocks;

// In-block prefix of scan block b for all kWalkThreads threads of the
// block: thread t holds master samples b·kWalkBlock + t·kWalkPer + i; on
// return v[i] is the thread's running sum and `offset` its exclusive prefix
// within the block, so P_b = offset ⊕ v[i]. warp_tot: kWalkThreads/32
// doubles of shared memory. Ends with the block synchronised.
__device__ __forceinline__ void walk_block_prefix(uint64_t seed, double sigma, int64_t b, double *warp_tot,
                                                  double v[kWalkPer], double &offset) {
    const int64_t base = b * kWalkBlock + (int64_t)threadIdx.x * kWalkPer;
    double run = 0.0;
#pragma unroll
    for (int i = 0; i < kWalkPer; i += 4) {
        double z[4];
        walk_increments4(seed, (base + i) >> 2, sigma, z);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            run = __dadd_rn(run, z[j]);
            v[i + j] = run;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double incl = run;  // warp inclusive scan of per-thread totals
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        double o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl = __dadd_rn(o, incl);
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    double wpre = 0.0;
    for (int w = 0; w < wid; ++w) wpre = __dadd_rn(wpre, warp_tot[w]);
    offset = __dadd_rn(wpre, __dsub_rn(incl, run));
    __syncthreads();  // warp_tot may be reused by the caller's next block
}

// Shared staging of one scan block's 4096 values, so that global stores
// run coalesced: thread t's run of kWalkPer values sits at row t (rows
// padded by one double against bank conflicts); element k of the block is
// walk_stage_at(k).
constexpr int kWalkStageLd = kWalkPer + 1;
constexpr int kWalkStageDoubles = kWalkThreads * kWalkStageLd;
__device__ __forceinline__ int walk_stage_at(int k) { return (k / kWalkPer) * kWalkStageLd + k % kWalkPer; }

// Inclusive warp scan in a fixed order (Hillis–Steele): lane l's result
// depends only on lanes 0..l.
__device__ __forceinline__ double warp_incl_scan(double v, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v = __dadd_rn(o, v);
    }
    return v;
}

// Sum of group h's kGroupBlocks totals in the fixed order; all
// kGroupThreads threads take part and receive it. sh: 33 doubles.
__device__ __forceinline__ double walk_group_sum(const double *__restrict__ tot, int64_t h, double *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double incl = warp_incl_scan(tot[h * kGroupBlocks + threadIdx.x], lane);
    if (lane == 31) sh[w] = incl;
    __syncthreads();
    if (w == 0) {
        const double x = warp_incl_scan(sh[lane], lane);
        if (lane == 31) sh[32] = x;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// carry(b) for the blocks b in [bA, bB] of group g (kGroupThreads threads,
// one block each). Needs the totals of every block below bB and the sums
// of groups below g_known in gsum. Stores the sum of group g when the group
// is complete below bB and not yet stored; with write_prior also the sums
// of groups [g_known, g) it computes on the way. sh: 65 doubles.
__device__ __forceinline__ void walk_group_carries(const double *__restrict__ tot, double *__restrict__ gsum,
                                                   int64_t g_known, int64_t bA, int64_t bB, int64_t g,
                                                   bool write_prior, double *__restrict__ carry, double *sh) {
    double c2 = 0.0;  // Σ of the sums of groups 0..g-1, in group order
    const int64_t stored = g < g_known ? g : g_known;
    for (int64_t h = 0; h < stored; ++h) c2 = __dadd_rn(c2, gsum[h]);
    for (int64_t h = stored; h < g; ++h) {
        const double s = walk_group_sum(tot, h, sh);
        c2 = __dadd_rn(c2, s);
        if (write_prior && threadIdx.x == 0) gsum[h] = s;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t b = g * kGroupBlocks + threadIdx.x;
    const double incl = warp_incl_scan(b < bB ? tot[b] : 0.0, lane);
    double excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 0.0;
    if (lane == 31) sh[w] = incl;
    __syncthreads();
    if (w == 0) {
        const double x = warp_incl_scan(sh[lane], lane);
        double e2 = __shfl_up_sync(0xffffffffu, x, 1);
        if (lane == 0) e2 = 0.0;
        sh[33 + lane] = e2;
        if (lane == 31 && (g + 1) * kGroupBlocks <= bB && g >= g_known) gsum[g] = x;
    }
    __syncthreads();
    if (b >= bA && b <= bB) carry[b] = __dadd_rn(__dadd_rn(c2, sh[33 + w]), excl);
    __syncthreads();
}

}  // namespace lpk
