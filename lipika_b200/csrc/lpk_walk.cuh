// lpk_walk.cuh — the device clock walk's scan block, shared by the
// single-band and batched paths so that both produce the same bits.
//
// The walk ε(k) = Σ_{j<=k} σ z_j (white frequency noise integrated at the
// master rate, ClockStream::advance_to, src/clock/mod.rs:299-307) is
// defined through fixed scan blocks of kWalkBlock master samples:
// ε(k) = carry(b) + P_b(k), with P_b the in-block inclusive prefix computed
// in one fixed parallel order and carry(b) the sequential sum of the totals
// of blocks 0..b-1. Nothing depends on how a band is chunked.
#pragma once

#include "lpk_device.cuh"

namespace lpk {

constexpr int64_t kWalkBlock = 4096;  // master samples per scan block
constexpr int kWalkThreads = 256;
constexpr int kWalkPer = (int)(kWalkBlock / kWalkThreads);  // 16

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
    for (int i = 0; i < kWalkPer; ++i) {
        run = __dadd_rn(run, walk_increment(seed, base + i, sigma));
        v[i] = run;
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

}  // namespace lpk
