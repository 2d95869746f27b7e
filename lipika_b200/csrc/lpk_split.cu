// lpk_split.cu — the split-precision fan-out of one band chunk (see
// lpk_split.cuh for the numerical design): k_split_anchor fits each
// (tile, transmitter), then k_band_split evaluates every band sample of the
// tile against the fits. Every launch shape of LPK_SPLIT_VARIANTS is
// compiled; the context picks one.
#include "lpk_internal.h"
#include "lpk_split.cuh"

namespace lpk {

static_assert(sizeof(AnchorRec) + sizeof(AnchorExt) == 400,
              "lpk_band_chunk_device_static sizes its record area for 400-byte (record, extension) pairs");

namespace {

// One block per anchor group (lpk_split.cuh): up to 32 tiles (one per
// lane) of up to 4 transmitters (one per warp); the band is a kernel
// parameter, the group's transmitters are staged in shared memory, and the
// records go out tile-major through shared memory.
// MOV: the band's receiver is on an orbit (compiled apart, as the fan-out).
template <bool MOV>
__global__ void __launch_bounds__(kAnchorThreads, LPK_ANCHOR_MINB)
k_split_anchor(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active, int32_t n_active,
               int64_t t0, int64_t n_tiles, int32_t tile_len, AnchorRec *__restrict__ recs,
               AnchorExt *__restrict__ exts) {
    __shared__ __align__(16) AnchorRec srec[kAnchorThreads];
    __shared__ __align__(16) DevTx stx[kAnchorGroupTx];
    const int64_t ntg = (n_tiles + kAnchorGroupTiles - 1) / kAnchorGroupTiles;
    const int64_t tile0 = (int64_t)(blockIdx.x % ntg) * kAnchorGroupTiles;
    const int k0 = (int)(blockIdx.x / ntg) * kAnchorGroupTx;
    const int nt = (int)(n_tiles - tile0 < kAnchorGroupTiles ? n_tiles - tile0 : kAnchorGroupTiles);
    const int nk = n_active - k0 < kAnchorGroupTx ? n_active - k0 : kAnchorGroupTx;
    stage_group_txs(txs, active + k0, nk, stx);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane < nt && w < nk) {
        const int64_t tile = tile0 + lane;
        const int64_t gs = (t0 + tile) * tile_len;  // absolute sample indices of the tile
        fit_anchor<MOV>(b, stx[w], gs, gs + tile_len - 1, false, srec[lane * kAnchorGroupTx + w],
                        exts + tile * n_active + k0 + w);
    }
    __syncthreads();
    store_group(srec, recs + tile0 * n_active + k0, nt, nk, n_active);
}

// One block per tile. MOV: the band's receiver is on an orbit (compiled
// apart, so the stationary kernels carry no receiver-orbit code).
template <int TILE, int THREADS, int MINB, bool DBG, bool UNOCC, bool ACC, bool MOV>
__global__ void __launch_bounds__(THREADS, MINB)
k_band_split(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active, int32_t n_active,
             int64_t t0, const AnchorRec *__restrict__ recs, const AnchorExt *__restrict__ exts,
             float2 *__restrict__ out, double *dbg_phase,
             double *dbg_temit, double *dbg_delay) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevTx *stx = reinterpret_cast<DevTx *>(smem_raw);
    AnchorRec *srec = reinterpret_cast<AnchorRec *>(smem_raw + sizeof(DevTx) * (size_t)n_active);
    const int64_t tile = blockIdx.x;
    stage_tile(txs, active, n_active, recs + tile * n_active, stx, srec, true);
    __syncthreads();
    const int64_t first = (t0 + tile) * TILE - b.i0;  // chunk index of the tile's first sample
    split_tile<TILE / THREADS, THREADS, DBG, UNOCC, ACC, MOV>(b, stx, srec, exts + tile * n_active, n_active, first,
                                                              out, dbg_phase, dbg_temit, dbg_delay);
}

using SplitKernel = void (*)(const DevBand, const DevTx *, const int32_t *, int32_t, int64_t, const AnchorRec *,
                             const AnchorExt *, float2 *, double *, double *, double *);

struct SplitShape {
    int tile, threads, minb;
    SplitKernel fast[2], fast_unocc[2], dbg[2], acc[2];  // [receiver on an orbit]; acc: accuracy mode
};

#define LPK_SPLIT_ENTRY(I, T, N, M)                                                                              \
    {T, N, M,                                                                                                    \
     {k_band_split<T, N, M, false, false, false, false>, k_band_split<T, N, M, false, false, false, true>},      \
     {k_band_split<T, N, M, false, true, false, false>, k_band_split<T, N, M, false, true, false, true>},        \
     {k_band_split<T, N, M, true, false, false, false>, k_band_split<T, N, M, true, false, false, true>},        \
     {k_band_split<T, N, M, false, false, true, false>, k_band_split<T, N, M, false, false, true, true>}},
const SplitShape kShapes[kSplitVariants] = {LPK_SPLIT_VARIANTS(LPK_SPLIT_ENTRY)};
#undef LPK_SPLIT_ENTRY

int64_t split_tiles(int64_t i0, int64_t n, int tile) { return n > 0 ? (i0 + n - 1) / tile - i0 / tile + 1 : 0; }

}  // namespace

bool split_variant_info(int v, int *tile, int *threads, int *minb) {
    if (v < 0 || v >= kSplitVariants) return false;
    if (tile) *tile = kShapes[v].tile;
    if (threads) *threads = kShapes[v].threads;
    if (minb) *minb = kShapes[v].minb;
    return true;
}

size_t split_recs_bytes(int variant, int64_t i0, int64_t n, int32_t n_active) {
    return (sizeof(AnchorRec) + sizeof(AnchorExt)) * (size_t)split_tiles(i0, n, kShapes[variant].tile) *
           (size_t)n_active;
}

cudaError_t launch_split_anchor(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                               int32_t n_active, void *d_recs, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    const SplitShape &sh = kShapes[variant];
    const int64_t t0 = b.i0 / sh.tile;
    const int64_t n_tiles = split_tiles(b.i0, b.n, sh.tile);
    const int64_t na = n_tiles * n_active;
    if (na <= 0) return cudaSuccess;
    AnchorRec *recs = (AnchorRec *)d_recs;
    AnchorExt *exts = (AnchorExt *)(recs + na);  // 16-byte aligned: sizeof(AnchorRec) is a multiple of 16
    const int64_t groups = (n_tiles + kAnchorGroupTiles - 1) / kAnchorGroupTiles *
                           ((n_active + kAnchorGroupTx - 1) / kAnchorGroupTx);
    (b.rx_kind == LPK_RX_KEPLER ? k_split_anchor<true> : k_split_anchor<false>)<<<
        (unsigned)groups, kAnchorThreads, 0, s>>>(
        b, d_tx, d_active, n_active, t0, n_tiles, sh.tile, recs, exts);
    return cudaGetLastError();
}

cudaError_t launch_split_fanout(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                                int32_t n_active, void *d_recs, float2 *d_out, double *dbg_phase, double *dbg_temit,
                                double *dbg_delay, cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    const SplitShape &sh = kShapes[variant];
    const int64_t t0 = b.i0 / sh.tile;
    const int64_t n_tiles = split_tiles(b.i0, b.n, sh.tile);
    const int64_t na = n_tiles * n_active;
    AnchorRec *recs = (AnchorRec *)d_recs;
    AnchorExt *exts = (AnchorExt *)(recs + na);
    const size_t smem = (sizeof(DevTx) + sizeof(AnchorRec)) * (size_t)n_active;
    const int mov = b.rx_kind == LPK_RX_KEPLER;
    SplitKernel kern = b.acc_stats ? sh.acc[mov]
                                   : (dbg_phase ? sh.dbg[mov] : (b.unocc_words ? sh.fast_unocc[mov] : sh.fast[mov]));
    if (smem > 40 * 1024) {  // leaves room for the kernel's static shared arrays
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<(unsigned)n_tiles, sh.threads, smem, s>>>(b, d_tx, d_active, n_active, t0, recs, exts, d_out,
                                                     dbg_phase, dbg_temit, dbg_delay);
    return cudaGetLastError();
}

cudaError_t launch_band_split(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                              int32_t n_active, void *d_recs, float2 *d_out, double *dbg_phase, double *dbg_temit,
                              double *dbg_delay, cudaStream_t s) {
    cudaError_t e = launch_split_anchor(variant, b, d_tx, d_active, n_active, d_recs, s);
    if (e != cudaSuccess) return e;
    return launch_split_fanout(variant, b, d_tx, d_active, n_active, d_recs, d_out, dbg_phase, dbg_temit, dbg_delay,
                               s);
}

}  // namespace lpk
