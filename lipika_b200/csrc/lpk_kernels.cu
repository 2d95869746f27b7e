// lpk_kernels.cu — the fan-out kernels.
//
// k_band_reference: one thread per band sample, the band's in-band
// transmitters in fixed order, each evaluated with the reference's exact
// f64 operation sequence (emission solve, s(t), mix), summed in f32 in
// transmitter order, then AWGN and the rx chain. This is the all-FP64 path
// that replaces src/pipeline.rs:943-983 bit-for-bit (up to the last ulp of
// CUDA's sin/cos).
#include "lpk_internal.h"
#include "lpk_contrib.cuh"
#include "lpk_walk.cuh"

namespace lpk {

namespace {

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock)
k_band_reference(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active,
                 int32_t n_active, float2 *__restrict__ out, uint32_t *__restrict__ unocc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevTx *stx = reinterpret_cast<DevTx *>(smem_raw);
    {
        const int words = (int)(sizeof(DevTx) / 8);
        for (int k = 0; k < n_active; ++k) {
            const uint64_t *src = reinterpret_cast<const uint64_t *>(txs + active[k]);
            uint64_t *dst = reinterpret_cast<uint64_t *>(stx + k);
            for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
        }
    }
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = j < b.n;
    const int64_t g = b.i0 + j;
    double t_local = 0.0, delta = 0.0, tu = 0.0, ox = 0.0, oy = 0.0, oz = 0.0;
    if (live) {
        t_local = __ddiv_rn((double)g, b.fs);  // src/pipeline.rs:918
        delta = band_delta(b, j, t_local);
        tu = __dsub_rn(t_local, delta);         // :927
        band_rx(b, j, tu, ox, oy, oz);
    }
    // Horizon gate over the block's samples (src/channel/horizon.rs): a
    // transmitter certainly below the antenna cutoff for all of them is
    // skipped; the per-sample path would give it zero gain everywhere.
    __shared__ double red[96];
    __shared__ unsigned char skip[256];
    // (a receiver on an orbit is not gated: the bound needs the block's
    // receiver positions before the solve; skipping is an optimisation only)
    const bool gate = b.has_antenna && b.has_cutoff && b.rx_kind != LPK_RX_KEPLER;
    if (gate) {
        double cx, cy, cz;
        band_rx(b, (int64_t)blockIdx.x * blockDim.x, 0.0, cx, cy, cz);  // the block's first sample is in the chunk
        double lo = live ? tu : __longlong_as_double(0x7ff0000000000000LL);
        double hi = live ? tu : -__longlong_as_double(0x7ff0000000000000LL);
        const double ex = ox - cx, ey = oy - cy, ez = oz - cz;
        double r2 = live ? ex * ex + ey * ey + ez * ez : 0.0;
        bool fin = !live || (isfinite(tu) && isfinite(r2));
        block_min_max_and(lo, hi, r2, fin, red);
        for (int k = threadIdx.x; k < n_active; k += blockDim.x) {
            const bool sk = fin && certainly_below_cutoff(stx[k], b.epoch, lo, hi, cx, cy, cz, sqrt(r2), b.ant_cutoff);
            skip[k] = sk;
            if (b.gate_stats) {
                atomicAdd(b.gate_stats, 1ull);
                if (sk) atomicAdd(b.gate_stats + 1, 1ull);
            }
        }
        __syncthreads();
    }
    float acc_re = 0.0f, acc_im = 0.0f;
    for (int k = 0; k < n_active; ++k) {
        if (gate && skip[k]) continue;  // block-uniform
        float cr = 0.0f, ci = 0.0f;
        bool on = false;
        if (live) {
            on = contribution(stx[k], b, t_local, tu, delta, ox, oy, oz, cr, ci, nullptr, nullptr, nullptr);
            if (on) {  // fixed-order Σ, pipeline.rs:966-977
                acc_re = __fadd_rn(acc_re, cr);
                acc_im = __fadd_rn(acc_im, ci);
            }
        }
        if (b.has_antenna && unocc) {
            unsigned any = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0 && any) atomicOr(unocc + k, 1u);
        }
    }
    if (!live) return;
    out[j] = band_epilogue(b, acc_re, acc_im, g);
}

// The tuned all-FP64 fan-out (contribution_fp64): one thread per band
// sample, the band's transmitters from shared memory in active-list order,
// the sample time as the IEEE quotient without a division sequence, the
// epilogue of k_band_reference. Within tolerance of k_band_reference.
__global__ void __launch_bounds__(kBlock)
k_band_fp64(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active, int32_t n_active,
            float2 *__restrict__ out, uint32_t *__restrict__ unocc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevTx *stx = reinterpret_cast<DevTx *>(smem_raw);
    {
        const int words = (int)(sizeof(DevTx) / 8);
        for (int k = 0; k < n_active; ++k) {
            const uint64_t *src = reinterpret_cast<const uint64_t *>(txs + active[k]);
            uint64_t *dst = reinterpret_cast<uint64_t *>(stx + k);
            for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
        }
    }
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = j < b.n;
    const int64_t g = b.i0 + (live ? j : 0);
    const double t_local = sample_time((double)g, b.fs, __drcp_rn(b.fs));
    const double delta = band_delta(b, live ? j : 0, t_local);
    const double tu = t_local - delta;
    double ox, oy, oz;
    band_rx(b, live ? j : 0, tu, ox, oy, oz);
    float acc_re = 0.0f, acc_im = 0.0f;
    for (int k = 0; k < n_active; ++k) {
        float cr = 0.0f, ci = 0.0f;
        const bool on = live && contribution_fp64(stx[k], b, t_local, tu, delta, ox, oy, oz, cr, ci);
        if (on) {
            acc_re = __fadd_rn(acc_re, cr);
            acc_im = __fadd_rn(acc_im, ci);
        }
        if (b.has_antenna && unocc) {
            unsigned any = __ballot_sync(0xffffffffu, on);
            if ((threadIdx.x & 31) == 0 && any) atomicOr(unocc + k, 1u);
        }
    }
    if (!live) return;
    out[j] = band_epilogue(b, acc_re, acc_im, g);
}

__global__ void __launch_bounds__(kBlock)
k_tx_contribution(const DevBand b, const DevTx *__restrict__ txs, int32_t tx_idx, float2 *__restrict__ out,
                  double *phase, double *temit, double *range) {
    __shared__ DevTx stx;
    if (threadIdx.x == 0) stx = txs[tx_idx];
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= b.n) return;
    const int64_t g = b.i0 + j;
    double t_local = __ddiv_rn((double)g, b.fs);
    double delta = band_delta(b, j, t_local);
    double tu = __dsub_rn(t_local, delta);
    double ox, oy, oz;
    band_rx(b, j, tu, ox, oy, oz);
    float cr = 0.0f, ci = 0.0f;
    contribution(stx, b, t_local, tu, delta, ox, oy, oz, cr, ci, phase ? phase + j : nullptr,
                 temit ? temit + j : nullptr, range ? range + j : nullptr);
    out[j] = make_float2(cr, ci);
}

__global__ void __launch_bounds__(kBlock)
k_solve(const DevTx *__restrict__ txs, int32_t tx_idx, const double *__restrict__ obs,
        const double *__restrict__ t, int64_t n, double epoch, int32_t iterations, double inv_c,
        double *__restrict__ temit, double *__restrict__ range) {
    __shared__ DevTx stx;
    if (threadIdx.x == 0) stx = txs[tx_idx];
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double te, r;
    solve_reference(stx, t[j], obs[j], obs[n + j], obs[2 * n + j], epoch, iterations, inv_c, te, r);
    temit[j] = te;
    range[j] = r;
}

__global__ void __launch_bounds__(kBlock)
k_rx_chain(const DevBand b, float2 *__restrict__ iq) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= b.n) return;
    float2 v = iq[j];
    iq[j] = band_epilogue(b, v.x, v.y, b.i0 + j);
}

// ---------------------------------------------------------------- clock walk
// One block per scan block (lpk_walk.cuh): its total (totals != NULL), or
// ε(k) = carry(b) ⊕ P_b(k) for the master indices [kA, kB] it holds.
__global__ void __launch_bounds__(kWalkThreads, LPK_WALK_MINB)
k_walk_block(uint64_t seed, double sigma, int64_t b0, double *__restrict__ totals,
             const double *__restrict__ carry, double *__restrict__ eps, int64_t kA, int64_t kB) {
    __shared__ double warp_tot[kWalkThreads / 32];
    __shared__ double stage[kWalkStageDoubles];
    const int64_t b = b0 + blockIdx.x;
    double v[kWalkPer], offset;
    walk_block_prefix(seed, sigma, b, warp_tot, v, offset);
    if (totals) {
        if (threadIdx.x == kWalkThreads - 1) totals[b] = __dadd_rn(offset, v[kWalkPer - 1]);
        return;
    }
    const double c = carry[b];
#pragma unroll
    for (int i = 0; i < kWalkPer; ++i)
        stage[threadIdx.x * kWalkStageLd + i] = __dadd_rn(c, __dadd_rn(offset, v[i]));
    __syncthreads();
    for (int kk = threadIdx.x; kk < (int)kWalkBlock; kk += kWalkThreads) {
        const int64_t k = b * kWalkBlock + kk;
        if (k >= kA && k <= kB) eps[k - kA] = stage[walk_stage_at(kk)];
    }
}

// carry(b) for b in [bA, bB], one block per carry group (lpk_walk.cuh).
__global__ void __launch_bounds__(kGroupThreads)
k_walk_carries(const double *__restrict__ tot, double *__restrict__ gsum, int64_t g_known, int64_t bA, int64_t bB,
               double *__restrict__ carry) {
    __shared__ double sh[65];
    const int64_t g = bA / kGroupBlocks + blockIdx.x;
    walk_group_carries(tot, gsum, g_known, bA, bB, g, blockIdx.x == 0, carry, sh);
}

// The split fan-out's sample times for indices i0 .. i0 + n - 1.
__global__ void __launch_bounds__(kBlock) k_sample_times(double fs, int64_t i0, int64_t n, double *__restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    out[j] = sample_time((double)(i0 + j), fs, __drcp_rn(fs));
}

__global__ void __launch_bounds__(kBlock) k_band_delta(const DevBand b, double *__restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= b.n) return;
    out[j] = band_delta(b, j, __ddiv_rn((double)(b.i0 + j), b.fs));
}

// unoccluded[k] |= flag: from the kernel's per-transmitter words (mode 0),
// or "at least one sample" without an antenna (mode 1), or nothing (mode 2).
__global__ void k_or_flags(const uint32_t *__restrict__ uw, uint8_t *__restrict__ unocc, int32_t n_active,
                           int mode) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_active) return;
    uint8_t f = mode == 0 ? (uint8_t)(uw[k] != 0) : (uint8_t)(mode == 1);
    unocc[k] |= f;
}

inline unsigned grid_for(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

namespace {
// Eight independent DFMA chains per thread, all in registers: issue-bound on
// the FP64 pipe. The result is stored so nothing is optimised away.
__global__ void __launch_bounds__(256) k_fp64_probe(double *out, int iters) {
    double a = 1.0 + threadIdx.x * 1e-9, b = 0.999999, c = 1e-7;
    double x0 = a, x1 = a + 1, x2 = a + 2, x3 = a + 3, x4 = a + 4, x5 = a + 5, x6 = a + 6, x7 = a + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, b, c); x1 = fma(x1, b, c); x2 = fma(x2, b, c); x3 = fma(x3, b, c);
        x4 = fma(x4, b, c); x5 = fma(x5, b, c); x6 = fma(x6, b, c); x7 = fma(x7, b, c);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace

cudaError_t launch_fp64_probe(double *d_out, int blocks, int iters, cudaStream_t s) {
    k_fp64_probe<<<blocks, 256, 0, s>>>(d_out, iters);
    return cudaGetLastError();
}

cudaError_t launch_sample_times(double fs, int64_t i0, int64_t n, double *d_out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_sample_times<<<grid_for(n), kBlock, 0, s>>>(fs, i0, n, d_out);
    return cudaGetLastError();
}

cudaError_t launch_band_delta(const DevBand &b, double *d_out, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    k_band_delta<<<grid_for(b.n), kBlock, 0, s>>>(b, d_out);
    return cudaGetLastError();
}

cudaError_t launch_or_flags(const uint32_t *d_uw, uint8_t *d_unocc, int32_t n_active, int mode, cudaStream_t s) {
    k_or_flags<<<1, 256, 0, s>>>(d_uw, d_unocc, n_active, mode);
    return cudaGetLastError();
}

cudaError_t launch_walk_totals(uint64_t seed, double sigma, int64_t b_from, int64_t b_to, double *d_tot,
                               cudaStream_t s) {
    if (b_to <= b_from) return cudaSuccess;
    k_walk_block<<<(unsigned)(b_to - b_from), kWalkThreads, 0, s>>>(seed, sigma, b_from, d_tot, nullptr, nullptr, 0,
                                                                     -1);
    return cudaGetLastError();
}

cudaError_t launch_walk_carries(const double *d_tot, double *d_gsum, int64_t g_known, int64_t bA, int64_t bB,
                                double *d_carry, cudaStream_t s) {
    if (bB < bA) return cudaSuccess;
    const int64_t groups = bB / kGroupBlocks - bA / kGroupBlocks + 1;
    k_walk_carries<<<(unsigned)groups, kGroupThreads, 0, s>>>(d_tot, d_gsum, g_known, bA, bB, d_carry);
    return cudaGetLastError();
}

cudaError_t launch_walk_materialize(uint64_t seed, double sigma, const double *d_carry, int64_t kA, int64_t kB,
                                    double *d_eps, cudaStream_t s) {
    if (kB < kA) return cudaSuccess;
    int64_t b0 = kA / kWalkBlock, b1 = kB / kWalkBlock;
    k_walk_block<<<(unsigned)(b1 - b0 + 1), kWalkThreads, 0, s>>>(seed, sigma, b0, nullptr, d_carry, d_eps, kA, kB);
    return cudaGetLastError();
}

cudaError_t launch_band_reference(const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                                  int32_t n_active, float2 *d_out, uint32_t *d_unocc, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    size_t smem = sizeof(DevTx) * (size_t)n_active;
    if (smem > 40 * 1024) {  // leaves room for the kernel's static shared arrays
        cudaError_t e = cudaFuncSetAttribute(k_band_reference, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_band_reference<<<grid_for(b.n), kBlock, smem, s>>>(b, d_tx, d_active, n_active, d_out, d_unocc);
    return cudaGetLastError();
}

cudaError_t launch_band_fp64(const DevBand &b, const DevTx *d_tx, const int32_t *d_active, int32_t n_active,
                             float2 *d_out, uint32_t *d_unocc, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    size_t smem = sizeof(DevTx) * (size_t)n_active;
    if (smem > 40 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_band_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_band_fp64<<<grid_for(b.n), kBlock, smem, s>>>(b, d_tx, d_active, n_active, d_out, d_unocc);
    return cudaGetLastError();
}

cudaError_t launch_tx_contribution(const DevBand &b, const DevTx *d_tx, int32_t tx, float2 *d_out,
                                   double *d_phase, double *d_temit, double *d_range, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    k_tx_contribution<<<grid_for(b.n), kBlock, 0, s>>>(b, d_tx, tx, d_out, d_phase, d_temit, d_range);
    return cudaGetLastError();
}

cudaError_t launch_rx_chain(const DevBand &b, float2 *d_iq, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    k_rx_chain<<<grid_for(b.n), kBlock, 0, s>>>(b, d_iq);
    return cudaGetLastError();
}

cudaError_t launch_solve(const DevTx *d_tx, int32_t tx, const double *d_obs, const double *d_t, int64_t n,
                         double epoch, int32_t iterations, double inv_c, double *d_temit, double *d_range,
                         cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_solve<<<grid_for(n), kBlock, 0, s>>>(d_tx, tx, d_obs, d_t, n, epoch, iterations, inv_c, d_temit, d_range);
    return cudaGetLastError();
}

}  // namespace lpk
