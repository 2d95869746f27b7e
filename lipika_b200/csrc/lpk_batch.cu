// lpk_batch.cu — every (receiver, band) work unit of a scene in one
// persistent fan-out per round, replayed as a CUDA graph.
//
// The reference renders each work unit with its own generate_band call
// (src/pipeline.rs:506-535, one rayon task per (rx, band)); each call
// regenerates its receiver's clock walk (src/pipeline.rs:864-873). Here a
// round advances every unit by the same stretch of time: one graph copies
// the round's descriptor, scans the clock walk of every receiver once (all
// bands of a receiver read it), fits the anchors of every (unit, tile,
// transmitter), and runs one persistent kernel whose blocks pull tiles of
// all units from a shared counter, so units of uneven rate, length and
// transmitter count keep every SM busy until the round's last tile.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lpk_internal.h"
#include "lpk_split.cuh"

namespace lpk {

namespace {

constexpr int kMaxUnits = 256;
constexpr int kMaxWalks = kMaxUnits;  // at most one walk per unit

// Per unit, fixed for the batch.
struct BatchUnit {
    int32_t act_off, n_active;
    int32_t walk;        // index into the walk table, -1 without a device walk
    int32_t exact_only;  // reference-exact path for every sample
    float2 *out[2];      // round output buffers (capacity: the unit's round length),
                         // alternating between rounds so one can be read while the next renders
};

// One receiver clock walk: the scan blocks' totals and carries over the
// whole scene, and the in-block prefixes of the current round.
struct DevWalk {
    uint64_t seed;
    double sigma;
    double *partial;  // P_b(k) for k in [bA·kWalkBlock, (bB+1)·kWalkBlock)
    double *totals;   // per scan block
    double *gsum;     // per carry group of kGroupBlocks scan blocks
    double *carry;    // carry[b] = Σ totals[0..b-1] in the fixed order of lpk_walk.cuh
};

// Per round (copied to the device by the graph's first node).
struct RoundUnit {
    int64_t i0, n;          // band samples [i0, i0 + n)
    int64_t t0, n_tiles;    // absolute index of the first tile, tile count
    int64_t tile_off, rec_off;  // prefix over schedule slots
    int64_t grp_off;            // prefix of anchor groups (lpk_split.cuh) over schedule slots
    int32_t unit, pad;
};
struct RoundWalk {
    int64_t b_lo, bA, bB;   // blocks [b_lo, bB] are scanned, P_b stored for [bA, bB]
    int64_t g_known;        // groups whose sums are stored before the round
};
struct RoundDesc {
    int64_t total_tiles, total_groups, total_walk_blocks;
    int32_t n_slots, n_walks, tile, parity;  // parity: which output buffer the round writes
    int64_t wb_off[kMaxWalks + 1];  // prefix of scanned blocks per walk
    RoundWalk w[kMaxWalks];
    RoundUnit s[kMaxUnits];         // schedule slots, most work first
};

__device__ __forceinline__ int find_slot_tiles(const RoundDesc &rd, int64_t g) {
    int lo = 0, hi = rd.n_slots - 1;
    while (lo < hi) {  // last slot with tile_off <= g
        int mid = (lo + hi + 1) >> 1;
        if (rd.s[mid].tile_off <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_slot_groups(const RoundDesc &rd, int64_t g) {
    int lo = 0, hi = rd.n_slots - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (rd.s[mid].grp_off <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Scan blocks of every walk of the round (grid-stride, one block per scan
// block): totals always, in-block prefixes for [bA, bB].
__global__ void __launch_bounds__(kWalkThreads, LPK_WALK_MINB)
k_batch_walk(const DevWalk *__restrict__ walks, const RoundDesc *__restrict__ rd) {
    __shared__ double warp_tot[kWalkThreads / 32];
    __shared__ double stage[kWalkStageDoubles];
    const int64_t total = rd->total_walk_blocks;
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        int w = 0;
        while (w + 1 < rd->n_walks && rd->wb_off[w + 1] <= g) ++w;
        const RoundWalk rw = rd->w[w];
        const DevWalk dw = walks[w];
        const int64_t b = rw.b_lo + (g - rd->wb_off[w]);
        double v[kWalkPer], offset;
        walk_block_prefix(dw.seed, dw.sigma, b, warp_tot, v, offset);
        if (threadIdx.x == kWalkThreads - 1) dw.totals[b] = __dadd_rn(offset, v[kWalkPer - 1]);
        if (b >= rw.bA) {  // block-uniform
#pragma unroll
            for (int i = 0; i < kWalkPer; ++i) stage[threadIdx.x * kWalkStageLd + i] = __dadd_rn(offset, v[i]);
            __syncthreads();
            double *dst = dw.partial + (b - rw.bA) * kWalkBlock;
            for (int kk = threadIdx.x; kk < (int)kWalkBlock; kk += kWalkThreads) dst[kk] = stage[walk_stage_at(kk)];
            __syncthreads();  // stage is rewritten by the next block
        }
    }
}

// Sums of the carry groups [g_known, bB / kGroupBlocks) of every walk (the
// groups the round completes), one block per group: blockIdx.y is the walk.
__global__ void __launch_bounds__(kGroupThreads)
k_batch_gsum(const DevWalk *__restrict__ walks, const RoundDesc *__restrict__ rd) {
    __shared__ double sh[33];
    const int w = (int)blockIdx.y;
    if (w >= rd->n_walks) return;
    const RoundWalk rw = rd->w[w];
    if (rw.bB < rw.bA) return;
    const DevWalk dw = walks[w];
    for (int64_t h = rw.g_known + blockIdx.x; h < rw.bB / kGroupBlocks; h += gridDim.x) {
        const double v = walk_group_sum(dw.totals, h, sh);
        if (threadIdx.x == 0) dw.gsum[h] = v;
    }
}

// Carries of the round's blocks [bA, bB] of every walk (lpk_walk.cuh), after
// k_batch_gsum has stored every group sum they need: blockIdx.y is the walk,
// blocks stride over its carry groups.
__global__ void __launch_bounds__(kGroupThreads)
k_batch_carry(const DevWalk *__restrict__ walks, const RoundDesc *__restrict__ rd) {
    __shared__ double sh[65];
    const int w = (int)blockIdx.y;
    if (w >= rd->n_walks) return;
    const RoundWalk rw = rd->w[w];
    if (rw.bB < rw.bA) return;
    const DevWalk dw = walks[w];
    const int64_t gA = rw.bA / kGroupBlocks, gB = rw.bB / kGroupBlocks;
    const int64_t known = gB > rw.g_known ? gB : rw.g_known;
    for (int64_t g = gA + blockIdx.x; g <= gB; g += gridDim.x)
        walk_group_carries(dw.totals, dw.gsum, known, rw.bA, rw.bB, g, false, dw.carry, sh);
}

// Anchor fits of every (slot, tile, transmitter) of the round by anchor
// groups (lpk_split.cuh): a block takes up to 32 tiles (one per lane) of up
// to 4 transmitters (one per warp) of one unit, stages the group's
// transmitters in shared memory (the band's fields are block-uniform reads),
// fits, and stores the records tile-major. The block's shared memory stays
// within the carveout that keeps five blocks per SM.
// MOV: some unit's receiver is on an orbit (compiled apart, as the fan-out).
template <bool MOV>
__global__ void __launch_bounds__(kAnchorThreads, LPK_ANCHOR_MINB)
k_batch_anchor(const DevBand *__restrict__ bands, const BatchUnit *__restrict__ units,
               const DevTx *__restrict__ txs, const int32_t *__restrict__ act, const RoundDesc *__restrict__ rd,
               AnchorRec *__restrict__ recs, AnchorExt *__restrict__ exts) {
    __shared__ __align__(16) AnchorRec srec[kAnchorThreads];
    __shared__ __align__(16) DevTx stx[kAnchorGroupTx];
    __shared__ int s_slot;
    const int tile_len = rd->tile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t g = blockIdx.x; g < rd->total_groups; g += gridDim.x) {
        if (threadIdx.x == 0) s_slot = find_slot_groups(*rd, g);
        __syncthreads();
        const RoundUnit &ru = rd->s[s_slot];
        const BatchUnit bu = units[ru.unit];
        const int64_t ntg = (ru.n_tiles + kAnchorGroupTiles - 1) / kAnchorGroupTiles, local = g - ru.grp_off;
        const int64_t tile0 = (local % ntg) * kAnchorGroupTiles;
        const int k0 = (int)(local / ntg) * kAnchorGroupTx;
        const int nt = (int)(ru.n_tiles - tile0 < kAnchorGroupTiles ? ru.n_tiles - tile0 : kAnchorGroupTiles);
        const int nk = bu.n_active - k0 < kAnchorGroupTx ? bu.n_active - k0 : kAnchorGroupTx;
        const DevBand &sb = bands[ru.unit];
        stage_group_txs(txs, act + bu.act_off + k0, nk, stx);
        __syncthreads();
        if (lane < nt && w < nk) {
            const int64_t tile = tile0 + lane;
            const int64_t gs = (ru.t0 + tile) * tile_len;
            AnchorExt *x = exts + ru.rec_off + tile * bu.n_active + k0 + w;
            if (MOV && sb.rx_kind == LPK_RX_KEPLER)
                fit_anchor<true>(sb, stx[w], gs, gs + tile_len - 1, bu.exact_only != 0,
                                 srec[lane * kAnchorGroupTx + w], x);
            else
                fit_anchor<false>(sb, stx[w], gs, gs + tile_len - 1, bu.exact_only != 0,
                                  srec[lane * kAnchorGroupTx + w], x);
        }
        __syncthreads();
        store_group(srec, recs + ru.rec_off + tile0 * bu.n_active + k0, nt, nk, bu.n_active);
        __syncthreads();  // srec and stx are rewritten by the next group
    }
}

// The persistent fan-out: blocks take tiles from the round's counter until
// none is left, claiming two tiles ahead (the claim's latency is hidden and
// the end-of-tile barrier publishes it), so one lane can ask for the next
// tile's anchor records to be brought into L2 while the current tile
// renders. A block restages the band and its transmitters only when the next
// tile belongs to another unit.
// MOV: some unit's receiver is on an orbit; its tiles take the orbit-aware
// tile code (compiled apart, so batches of stationary receivers run kernels
// without it). OOL: the exact path is an out-of-line call (batches with a
// split unit, whose exact samples are rare; a batch of reference-solver units
// only keeps it inline).
template <int TILE, int THREADS, int MINB, bool MOV, bool OOL>
__global__ void __launch_bounds__(THREADS, MINB)
k_batch_fanout(const DevBand *__restrict__ bands, const BatchUnit *__restrict__ units,
               const DevTx *__restrict__ txs, const int32_t *__restrict__ act, const DevWalk *__restrict__ walks,
               const RoundDesc *__restrict__ rd, const AnchorRec *__restrict__ recs,
               const AnchorExt *__restrict__ exts, unsigned long long *__restrict__ counter, int32_t max_active) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevBand *sb = reinterpret_cast<DevBand *>(smem_raw);
    DevTx *stx = reinterpret_cast<DevTx *>(smem_raw + ((sizeof(DevBand) + 15) / 16) * 16);
    AnchorRec *srec = reinterpret_cast<AnchorRec *>(reinterpret_cast<unsigned char *>(stx) +
                                                    sizeof(DevTx) * (size_t)max_active);
    __shared__ unsigned long long s_next[3];  // tiles it, it + 1 (published) and it + 2 (being claimed)
    int cur = -1;
    const int64_t total = rd->total_tiles;
    if (threadIdx.x == 0) {
        s_next[0] = atomicAdd(counter, 1ull);
        s_next[1] = atomicAdd(counter, 1ull);
    }
    __syncthreads();
    for (int it = 0;; ++it) {
        const int64_t g = (int64_t)s_next[it % 3];
        if (g >= total) break;
        if (threadIdx.x == 0) s_next[(it + 2) % 3] = atomicAdd(counter, 1ull);  // read after the end-of-tile barrier
        if (threadIdx.x == 32) {  // the next tile's records into L2 while this tile renders (no completion to wait on)
            const int64_t gn = (int64_t)s_next[(it + 1) % 3];
            if (gn < total) {
                const RoundUnit &rn = rd->s[find_slot_tiles(*rd, gn)];
                const int na = units[rn.unit].n_active;
                if (na > 0)
                    prefetch_l2(recs + rn.rec_off + (gn - rn.tile_off) * na, (uint32_t)(sizeof(AnchorRec) * na));
            }
        }
        const int sl = find_slot_tiles(*rd, g);
        const RoundUnit &ru = rd->s[sl];
        const BatchUnit bu = units[ru.unit];
        const int64_t local = g - ru.tile_off;
        const bool fresh = ru.unit != cur;
        if (fresh && threadIdx.x == 0) {
            DevBand b = bands[ru.unit];
            b.i0 = ru.i0;
            b.n = ru.n;
            if (bu.walk >= 0) {
                b.eps = walks[bu.walk].partial;
                b.eps_carry = walks[bu.walk].carry;
                b.eps_k0 = rd->w[bu.walk].bA * kWalkBlock;
            }
            *sb = b;
        }
        stage_tile(txs, act + bu.act_off, bu.n_active, recs + ru.rec_off + local * bu.n_active, stx, srec, fresh);
        cur = ru.unit;
        __syncthreads();
        const int64_t first = (ru.t0 + local) * TILE - ru.i0;
        const AnchorExt *xrec = exts + ru.rec_off + local * bu.n_active;
        if (MOV && sb->rx_kind == LPK_RX_KEPLER)  // block-uniform
            split_tile<TILE / THREADS, THREADS, false, false, false, true, OOL>(
                *sb, stx, srec, xrec, bu.n_active, first, bu.out[rd->parity], nullptr, nullptr, nullptr);
        else
            split_tile<TILE / THREADS, THREADS, false, false, false, false, OOL>(
                *sb, stx, srec, xrec, bu.n_active, first, bu.out[rd->parity], nullptr, nullptr, nullptr);
        __syncthreads();  // the next stage overwrites the shared tiles
    }
}

using FanoutKernel = void (*)(const DevBand *, const BatchUnit *, const DevTx *, const int32_t *, const DevWalk *,
                              const RoundDesc *, const AnchorRec *, const AnchorExt *, unsigned long long *,
                              int32_t);

struct FanoutShape {
    int tile, threads;
    FanoutKernel kern[2][2];  // [some receiver on an orbit][some unit on the split solver]
};
#define LPK_BATCH_ENTRY(I, T, N, M)                                                                    \
    {T, N, {{k_batch_fanout<T, N, M, false, false>, k_batch_fanout<T, N, M, false, true>},           \
            {k_batch_fanout<T, N, M, true, false>, k_batch_fanout<T, N, M, true, true>}}},
const FanoutShape kFanout[kSplitVariants] = {LPK_SPLIT_VARIANTS(LPK_BATCH_ENTRY)};
#undef LPK_BATCH_ENTRY

inline size_t fanout_smem(int max_active) {
    return ((sizeof(DevBand) + 15) / 16) * 16 + (sizeof(DevTx) + sizeof(AnchorRec)) * (size_t)max_active;
}

}  // namespace
}  // namespace lpk

using namespace lpk;

struct UnitHost {
    lpk_band_desc desc;
    int64_t n_samples = 0, round_len = 0;
    int32_t n_active = 0, walk = -1;
    bool exact_only = false;
};

struct WalkHost {
    uint64_t seed = 0;
    double fm = 0.0, sigma = 0.0;
    int64_t totals_done = 0;  // totals of blocks below this are known
    int64_t g_known = 0;      // sums of groups below this are stored
    int64_t partial_cap = 0;
};

struct lpk_batch {
    lpk_ctx *ctx = nullptr;
    std::vector<UnitHost> units;
    std::vector<WalkHost> walks;
    std::vector<void *> allocs;
    DevBand *d_bands = nullptr;
    BatchUnit *d_units = nullptr;
    std::vector<BatchUnit> h_units;
    int32_t *d_act = nullptr;
    DevWalk *d_walks = nullptr;
    RoundDesc *d_round = nullptr;
    RoundDesc *h_round[2] = {nullptr, nullptr};  // pinned, alternating between rounds
    cudaEvent_t done[2] = {nullptr, nullptr};       // round of parity p finished
    cudaEvent_t copied[2] = {nullptr, nullptr};     // output copies of parity p finished
    cudaStream_t side = nullptr;                    // graph branch: anchors beside the walk scan
    cudaStream_t copy = nullptr;                    // device-to-host copies of finished rounds
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t mark[2] = {nullptr, nullptr};       // placeholders of the profiling event nodes
    AnchorRec *d_recs = nullptr;
    AnchorExt *d_exts = nullptr;
    unsigned long long *d_counter = nullptr;
    int64_t recs_cap = 0;
    int64_t n_rounds = 0;
    int32_t max_active = 0;
    int any_orbit = 0;                              // some unit's receiver is on an orbit
    int any_split = 0;                              // some unit takes the split solver
    int variant = 0, bps = 0, max_bps = 0, walk_grid = 0, anchor_grid = 0;
    cudaGraph_t graph_src[2] = {nullptr, nullptr};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_prof[2] = {false, false};            // built with event nodes around the fan-out
    cudaGraphNode_t prof_node[2][2] = {};
    int parity = 0, last_parity = 0;
    int64_t last_round = -1;
    bool kit_complete = false;                      // every stream, event and descriptor above exists
    std::vector<lpk_cf32 *> staging[2];             // pinned host copies (lpk_batch_render), in the
                                                    // context's pinned pool
};

namespace {

lpk_status batch_alloc(lpk_batch *b, void **p, size_t bytes) {
    cudaError_t e = pool_alloc(b->ctx, p, bytes);
    if (e != cudaSuccess) return fail(b->ctx, LPK_ENOMEM, std::string("batch allocation failed: ") +
                                                                cudaGetErrorString(e));
    b->allocs.push_back(*p);
    return LPK_OK;
}

void unit_extent(const lpk_batch *b, int64_t round, int u, int64_t &i0, int64_t &n) {
    const UnitHost &uh = b->units[u];
    i0 = round * uh.round_len;
    n = uh.n_samples - i0;
    n = n < 0 ? 0 : (n > uh.round_len ? uh.round_len : n);
}

// Fill the round descriptor: schedule slots (most work first), tile and
// anchor prefixes for tile length `tile`, and the walk block ranges. With
// commit, the walks' carry bookkeeping advances.
void plan_round(lpk_batch *b, int64_t round, int tile, RoundDesc &rd, bool commit, int64_t *recs_out,
                int64_t *partial_blocks_out) {
    memset(&rd, 0, offsetof(RoundDesc, s));
    rd.tile = tile;
    std::vector<int> order;
    for (int u = 0; u < (int)b->units.size(); ++u) {
        int64_t i0, n;
        unit_extent(b, round, u, i0, n);
        if (n > 0) order.push_back(u);
    }
    auto cost = [&](int u) {
        int64_t i0, n;
        unit_extent(b, round, u, i0, n);
        return (double)n * (double)(b->units[u].n_active + 1);
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
    int64_t tiles = 0, recs = 0, groups = 0;
    std::vector<int64_t> kA(b->walks.size(), INT64_MAX), kB(b->walks.size(), -1);
    for (size_t sl = 0; sl < order.size(); ++sl) {
        const int u = order[sl];
        const UnitHost &uh = b->units[u];
        RoundUnit &ru = rd.s[sl];
        unit_extent(b, round, u, ru.i0, ru.n);
        ru.t0 = ru.i0 / tile;
        ru.n_tiles = (ru.i0 + ru.n - 1) / tile - ru.t0 + 1;
        ru.tile_off = tiles;
        ru.rec_off = recs;
        ru.grp_off = groups;
        ru.unit = u;
        tiles += ru.n_tiles;
        recs += ru.n_tiles * uh.n_active;
        groups += (ru.n_tiles + kAnchorGroupTiles - 1) / kAnchorGroupTiles *
                  ((uh.n_active + kAnchorGroupTx - 1) / kAnchorGroupTx);
        if (uh.walk >= 0) {
            int64_t a;
            int64_t span = walk_span(&uh.desc, ru.i0, ru.n, &a);
            kA[uh.walk] = std::min(kA[uh.walk], a);
            kB[uh.walk] = std::max(kB[uh.walk], a + span - 1);
        }
    }
    rd.n_slots = (int32_t)order.size();
    rd.total_tiles = tiles;
    rd.total_groups = groups;
    rd.n_walks = (int32_t)b->walks.size();
    int64_t wb = 0, partial_blocks = 0;
    for (size_t w = 0; w < b->walks.size(); ++w) {
        RoundWalk &rw = rd.w[w];
        WalkHost &wh = b->walks[w];
        rd.wb_off[w] = wb;
        if (kB[w] < 0) {  // no unit of this walk renders in this round
            rw.b_lo = rw.bA = 0;
            rw.bB = -1;
            rw.g_known = wh.g_known;
            continue;
        }
        rw.bA = kA[w] / kWalkBlock;
        rw.bB = kB[w] / kWalkBlock;
        rw.b_lo = std::min(rw.bA, wh.totals_done);
        rw.g_known = wh.g_known;
        wb += rw.bB - rw.b_lo + 1;
        partial_blocks = std::max(partial_blocks, rw.bB - rw.bA + 1);
        if (commit) {
            wh.totals_done = std::max(wh.totals_done, rw.bB + 1);
            wh.g_known = std::max(wh.g_known, rw.bB / kGroupBlocks);
        }
    }
    rd.wb_off[b->walks.size()] = wb;
    rd.total_walk_blocks = wb;
    if (recs_out) *recs_out = recs;
    if (partial_blocks_out) *partial_blocks_out = partial_blocks;
}

void drop_graphs(lpk_batch *b) {
    for (int p = 0; p < 2; ++p) {
        if (b->graph[p]) cudaGraphExecDestroy(b->graph[p]);
        if (b->graph_src[p]) cudaGraphDestroy(b->graph_src[p]);
        b->graph[p] = nullptr;
        b->graph_src[p] = nullptr;
    }
}

// Capture the round graph for the current launch configuration: the copy of
// descriptor h_round[p]; then, in parallel, the anchor fits (side branch)
// and the walk scan with its carries; then the counter reset and the
// persistent fan-out. With profiling on, two event-record nodes bracket the
// fan-out; each launch points them at a fresh event pair of the context.
lpk_status build_graph(lpk_batch *b, int p) {
    lpk_ctx *c = b->ctx;
    const FanoutShape &sh = kFanout[b->variant];
    const size_t smem = fanout_smem(b->max_active);
    const FanoutKernel kern = sh.kern[b->any_orbit][b->any_split];
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch fan-out shared memory");
    int dev_sms = 0;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    const bool prof = c->profiling;
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch graph capture");
    cudaMemcpyAsync(b->d_round, b->h_round[p], sizeof(RoundDesc), cudaMemcpyHostToDevice, c->stream);
    cudaEventRecord(b->fork, c->stream);
    cudaStreamWaitEvent(b->side, b->fork, 0);
    (b->any_orbit ? k_batch_anchor<true> : k_batch_anchor<false>)<<<b->anchor_grid, kAnchorThreads, 0, b->side>>>(
        b->d_bands, b->d_units, c->d_tx, b->d_act, b->d_round, b->d_recs, b->d_exts);
    cudaEventRecord(b->join, b->side);
    if (!b->walks.empty()) {
        k_batch_walk<<<b->walk_grid, kWalkThreads, 0, c->stream>>>(b->d_walks, b->d_round);
        k_batch_gsum<<<dim3(16, (unsigned)b->walks.size()), kGroupThreads, 0, c->stream>>>(b->d_walks, b->d_round);
        k_batch_carry<<<dim3(16, (unsigned)b->walks.size()), kGroupThreads, 0, c->stream>>>(b->d_walks, b->d_round);
    }
    cudaStreamWaitEvent(c->stream, b->join, 0);
    cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), c->stream);
    if (prof) cudaEventRecordWithFlags(b->mark[0], c->stream, cudaEventRecordExternal);
    kern<<<(unsigned)(dev_sms * b->bps), sh.threads, smem, c->stream>>>(
        b->d_bands, b->d_units, c->d_tx, b->d_act, b->d_walks, b->d_round, b->d_recs, b->d_exts, b->d_counter,
        b->max_active);
    if (prof) cudaEventRecordWithFlags(b->mark[1], c->stream, cudaEventRecordExternal);
    cudaError_t le = cudaGetLastError();
    e = cudaStreamEndCapture(c->stream, &g);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(c, le != cudaSuccess ? le : e, "batch graph capture");
    }
    b->graph_prof[p] = prof;
    if (prof) {  // find the two event-record nodes by their placeholder events
        size_t n = 0;
        cudaGraphGetNodes(g, nullptr, &n);
        std::vector<cudaGraphNode_t> nodes(n);
        cudaGraphGetNodes(g, nodes.data(), &n);
        b->prof_node[p][0] = b->prof_node[p][1] = nullptr;
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            cudaEvent_t ev = nullptr;
            if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeEventRecord) continue;
            if (cudaGraphEventRecordNodeGetEvent(nd, &ev) != cudaSuccess) continue;
            for (int k = 0; k < 2; ++k)
                if (ev == b->mark[k]) b->prof_node[p][k] = nd;
        }
        if (!b->prof_node[p][0] || !b->prof_node[p][1]) {
            cudaGraphDestroy(g);
            return fail(c, LPK_ECUDA, "profiling nodes missing from the round graph");
        }
    }
    e = cudaGraphInstantiate(&b->graph[p], g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        b->graph[p] = nullptr;
        return cuda_fail(c, e, "batch graph instantiate");
    }
    b->graph_src[p] = g;
    return LPK_OK;
}

lpk_status configure(lpk_batch *b, int variant, int bps) {
    if (variant < 0 || variant >= kSplitVariants) return fail(b->ctx, LPK_EINVAL, "unknown split variant");
    const FanoutShape &sh = kFanout[variant];
    const size_t smem = fanout_smem(b->max_active);
    const FanoutKernel kern = sh.kern[b->any_orbit][b->any_split];
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(b->ctx, e, "batch fan-out shared memory");
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, sh.threads, smem);
    if (e != cudaSuccess) return cuda_fail(b->ctx, e, "batch occupancy query");
    if (occ < 1) return fail(b->ctx, LPK_EINVAL, "batch fan-out does not fit on an SM");
    if (bps < 0) return fail(b->ctx, LPK_EINVAL, "blocks per SM must be >= 0");
    drop_graphs(b);
    b->variant = variant;
    b->max_bps = occ;
    b->bps = (bps == 0 || bps > occ) ? occ : bps;
    return LPK_OK;
}

}  // namespace

namespace lpk {
void batch_kit_destroy(BatchKit *k) {
    if (!k) return;
    for (void *h : k->h_round)
        if (h) cudaFreeHost(h);
    for (int i = 0; i < 2; ++i)
        for (cudaEvent_t ev : {k->done[i], k->copied[i], k->mark[i]})
            if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : {k->fork, k->join})
        if (ev) cudaEventDestroy(ev);
    for (cudaStream_t st : {k->side, k->copy})
        if (st) cudaStreamDestroy(st);
    delete k;
}
}  // namespace lpk

extern "C" {

int32_t lpk_split_variant_count(void) { return kSplitVariants; }

lpk_status lpk_split_variant_info(int32_t v, int32_t *tile, int32_t *threads, int32_t *min_blocks) {
    int t = 0, n = 0, m = 0;
    if (!split_variant_info(v, &t, &n, &m)) return fail(nullptr, LPK_EINVAL, "unknown split variant");
    if (tile) *tile = t;
    if (threads) *threads = n;
    if (min_blocks) *min_blocks = m;
    return LPK_OK;
}

lpk_status lpk_ctx_set_split_variant(lpk_ctx *c, int32_t v) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (v < 0 || v >= kSplitVariants) return fail(c, LPK_EINVAL, "unknown split variant");
    c->split_variant = v;
    return LPK_OK;
}

int32_t lpk_ctx_split_variant(const lpk_ctx *c) { return c ? c->split_variant : -1; }

void lpk_batch_destroy(lpk_batch *b) {
    if (!b) return;
    if (b->ctx) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
    }
    if (b->copy) cudaStreamSynchronize(b->copy);
    drop_graphs(b);
    for (void *p : b->allocs) pool_free(b->ctx, p);
    BatchKit *k = new BatchKit();
    for (int i = 0; i < 2; ++i) {
        k->h_round[i] = b->h_round[i];
        k->done[i] = b->done[i];
        k->copied[i] = b->copied[i];
        k->mark[i] = b->mark[i];
    }
    k->fork = b->fork;
    k->join = b->join;
    k->side = b->side;
    k->copy = b->copy;
    if (b->ctx && !b->ctx->batch_kit && b->kit_complete) b->ctx->batch_kit = k;  // the next batch reuses it
    else batch_kit_destroy(k);
    delete b;
}

lpk_status lpk_batch_create(lpk_ctx *c, const lpk_work_unit *wu, int32_t n_units, double round_s, lpk_batch **out) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (!out) return fail(c, LPK_EINVAL, "out is NULL");
    *out = nullptr;
    if (n_units < 1 || n_units > kMaxUnits) return fail(c, LPK_EINVAL, "batch needs 1..256 work units");
    if (!wu) return fail(c, LPK_EINVAL, "units is NULL");
    if (!(round_s > 0.0) || !std::isfinite(round_s)) return fail(c, LPK_EINVAL, "round_s must be positive");
    cudaSetDevice(c->device);
    lpk_batch *b = new lpk_batch();
    b->ctx = c;
    std::vector<DevBand> h_bands((size_t)n_units);
    std::vector<int32_t> h_act;
    lpk_status st = LPK_OK;
    for (int u = 0; u < n_units && !st; ++u) {
        const lpk_work_unit &w = wu[u];
        UnitHost uh;
        uh.desc = w.band;
        uh.n_samples = w.n_samples;
        uh.n_active = w.n_active;
        if (w.n_samples < 0) st = fail(c, LPK_EINVAL, "work unit length must be >= 0");
        else if (w.band.rx_kind != LPK_RX_STATIONARY && w.band.rx_kind != LPK_RX_KEPLER)
            st = fail(c, LPK_ENOTSUP, "batch units need a stationary or orbiting receiver (not per-sample positions)");
        else if (w.band.clock_mode != LPK_CLOCK_DETERMINISTIC && w.band.clock_mode != LPK_CLOCK_DEVICE_WALK)
            st = fail(c, LPK_ENOTSUP, "batch units need a deterministic or device-walk clock");
        else if ((st = build_dev_band(c, &w.band, 0, w.n_samples, h_bands[u]))) {
        } else if ((st = check_active(c, w.active, w.n_active))) {
        }
        if (st) break;
        uh.round_len = std::max<int64_t>(1, std::llround(round_s * w.band.fs_hz));
        uh.exact_only = !(w.band.solver == LPK_SOLVER_SPLIT);
        if (w.band.clock_mode == LPK_CLOCK_DEVICE_WALK) {
            const double sigma = w.band.clock_allan_1s / std::sqrt(w.band.clock_master_rate_hz);
            int found = -1;
            for (size_t k = 0; k < b->walks.size(); ++k)
                if (b->walks[k].seed == w.band.clock_seed && b->walks[k].fm == w.band.clock_master_rate_hz &&
                    b->walks[k].sigma == sigma)
                    found = (int)k;
            if (found < 0) {
                WalkHost wh;
                wh.seed = w.band.clock_seed;
                wh.fm = w.band.clock_master_rate_hz;
                wh.sigma = sigma;
                b->walks.push_back(wh);
                found = (int)b->walks.size() - 1;
            }
            uh.walk = found;
            h_bands[u].fm = w.band.clock_master_rate_hz;
        }
        BatchUnit bu{};
        bu.act_off = (int32_t)h_act.size();
        bu.n_active = w.n_active;
        bu.walk = uh.walk;
        bu.exact_only = uh.exact_only;
        for (int k = 0; k < w.n_active; ++k) h_act.push_back(w.active[k]);
        b->max_active = std::max(b->max_active, w.n_active);
        if (w.band.rx_kind == LPK_RX_KEPLER) b->any_orbit = 1;
        if (w.band.solver == LPK_SOLVER_SPLIT) b->any_split = 1;
        b->units.push_back(uh);
        b->h_units.push_back(bu);
    }
    if (st) {
        lpk_batch_destroy(b);
        return st;
    }
    for (auto &uh : b->units) {
        int64_t r = (uh.n_samples + uh.round_len - 1) / uh.round_len;
        b->n_rounds = std::max(b->n_rounds, r);
    }
    // capacities: anchors at the smallest tile, walk prefixes, scene-long carries
    RoundDesc *tmp = new RoundDesc();
    std::vector<WalkHost> saved = b->walks;
    for (int64_t r = 0; r < b->n_rounds; ++r) {
        int64_t recs = 0, pb = 0;
        plan_round(b, r, kSplitMinTile, *tmp, true, &recs, &pb);
        b->recs_cap = std::max(b->recs_cap, recs);
        for (auto &wh : b->walks) wh.partial_cap = std::max(wh.partial_cap, pb * kWalkBlock);
    }
    std::vector<int64_t> total_blocks(b->walks.size(), 1);
    for (size_t w = 0; w < b->walks.size(); ++w) {
        total_blocks[w] = b->walks[w].totals_done + 2;
        saved[w].partial_cap = b->walks[w].partial_cap;
    }
    b->walks = saved;  // carry bookkeeping restarts at block 0
    delete tmp;
    void *p = nullptr;
    if (!st) st = batch_alloc(b, &p, sizeof(DevBand) * (size_t)n_units), b->d_bands = (DevBand *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(BatchUnit) * (size_t)n_units), b->d_units = (BatchUnit *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(int32_t) * std::max<size_t>(1, h_act.size())), b->d_act = (int32_t *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(RoundDesc)), b->d_round = (RoundDesc *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(AnchorRec) * (size_t)std::max<int64_t>(1, b->recs_cap)),
             b->d_recs = (AnchorRec *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(AnchorExt) * (size_t)std::max<int64_t>(1, b->recs_cap)),
             b->d_exts = (AnchorExt *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(unsigned long long)), b->d_counter = (unsigned long long *)p;
    if (!st) st = batch_alloc(b, &p, sizeof(DevWalk) * std::max<size_t>(1, b->walks.size())),
             b->d_walks = (DevWalk *)p;
    for (int u = 0; u < n_units && !st; ++u)
        for (int k = 0; k < 2 && !st; ++k) {
            st = batch_alloc(b, &p, sizeof(float2) * (size_t)b->units[u].round_len);
            b->h_units[u].out[k] = (float2 *)p;
        }
    std::vector<DevWalk> h_walks(b->walks.size());
    for (size_t w = 0; w < b->walks.size() && !st; ++w) {
        h_walks[w].seed = b->walks[w].seed;
        h_walks[w].sigma = b->walks[w].sigma;
        st = batch_alloc(b, &p, sizeof(double) * (size_t)std::max<int64_t>(1, b->walks[w].partial_cap));
        h_walks[w].partial = (double *)p;
        if (!st) st = batch_alloc(b, &p, sizeof(double) * (size_t)total_blocks[w]), h_walks[w].totals = (double *)p;
        if (!st)
            st = batch_alloc(b, &p, sizeof(double) * (size_t)(total_blocks[w] + 1)), h_walks[w].carry = (double *)p;
        if (!st) st = batch_alloc(b, &p, sizeof(double) * (size_t)(total_blocks[w] / kGroupBlocks + 1)),
                 h_walks[w].gsum = (double *)p;
    }
    for (int u = 0; u < n_units && !st; ++u) {  // flicker tracks: each unit's whole track, uploaded once
        const lpk_band_desc &d = b->units[u].desc;
        if (!d.flicker_delta_s) continue;
        const int64_t last = b->units[u].n_samples > 0 ? b->units[u].n_samples - 1 : 0;
        const double x = ((double)last / d.fs_hz) * kFlickerRate;
        if ((x > 0.0 ? (int64_t)std::floor(x) : 0) + 1 >= d.flicker_n) {
            st = fail(c, LPK_EINVAL, "flicker track shorter than the work unit");
            break;
        }
        st = batch_alloc(b, &p, sizeof(double) * (size_t)d.flicker_n);
        if (st) break;
        cudaError_t e = cudaMemcpyAsync(p, d.flicker_delta_s, sizeof(double) * (size_t)d.flicker_n,
                                        cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) st = cuda_fail(c, e, "flicker track upload");
        h_bands[u].flicker = (const double *)p;
        h_bands[u].flicker_m0 = 0;
        h_bands[u].flicker_n = d.flicker_n;
    }
    if (!st && c->batch_kit) {  // streams, events and pinned descriptors of the last batch
        BatchKit *k = c->batch_kit;
        c->batch_kit = nullptr;
        for (int i = 0; i < 2; ++i) {
            b->h_round[i] = (RoundDesc *)k->h_round[i];
            b->done[i] = k->done[i];
            b->copied[i] = k->copied[i];
            b->mark[i] = k->mark[i];
        }
        b->fork = k->fork;
        b->join = k->join;
        b->side = k->side;
        b->copy = k->copy;
        delete k;
    } else {
        for (int i = 0; i < 2 && !st; ++i) {
            if (cudaHostAlloc((void **)&b->h_round[i], sizeof(RoundDesc), cudaHostAllocDefault) != cudaSuccess)
                st = fail(c, LPK_ENOMEM, "pinned round descriptor allocation failed");
            else if (cudaEventCreateWithFlags(&b->done[i], cudaEventDisableTiming) != cudaSuccess ||
                     cudaEventCreateWithFlags(&b->copied[i], cudaEventDisableTiming) != cudaSuccess ||
                     cudaEventCreate(&b->mark[i]) != cudaSuccess)
                st = fail(c, LPK_ECUDA, "event creation failed");
        }
        if (!st && (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
                    cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking) != cudaSuccess ||
                    cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess))
            st = fail(c, LPK_ECUDA, "stream or event creation failed");
    }
    if (!st) b->kit_complete = true;
    if (!st) {
        cudaError_t e = cudaMemcpyAsync(b->d_bands, h_bands.data(), sizeof(DevBand) * (size_t)n_units,
                                        cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->d_units, b->h_units.data(), sizeof(BatchUnit) * (size_t)n_units,
                                cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess && !h_act.empty())
            e = cudaMemcpyAsync(b->d_act, h_act.data(), sizeof(int32_t) * h_act.size(), cudaMemcpyHostToDevice,
                                c->stream);
        if (e == cudaSuccess && !h_walks.empty())
            e = cudaMemcpyAsync(b->d_walks, h_walks.data(), sizeof(DevWalk) * h_walks.size(), cudaMemcpyHostToDevice,
                                c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) st = cuda_fail(c, e, "batch upload");
    }
    if (!st) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        b->walk_grid = sms * 8;
        b->anchor_grid = sms * 8;
        st = configure(b, c->split_variant, 0);
    }
    if (st) {
        lpk_batch_destroy(b);
        return st;
    }
    *out = b;
    return LPK_OK;
}

int64_t lpk_batch_n_rounds(const lpk_batch *b) { return b ? b->n_rounds : -1; }

lpk_status lpk_batch_round_extent(const lpk_batch *b, int64_t round, int32_t unit, int64_t *i0, int64_t *n) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    if (unit < 0 || unit >= (int32_t)b->units.size()) return fail(b->ctx, LPK_EINVAL, "unit out of range");
    if (round < 0) return fail(b->ctx, LPK_EINVAL, "round must be >= 0");
    int64_t a, m;
    unit_extent(b, round, unit, a, m);
    if (i0) *i0 = a;
    if (n) *n = m;
    return LPK_OK;
}

lpk_status lpk_batch_run(lpk_batch *b, int64_t round) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    lpk_ctx *c = b->ctx;
    if (round < 0 || round >= b->n_rounds) return fail(c, LPK_EINVAL, "round out of range");
    cudaSetDevice(c->device);
    const int p = b->parity;
    // descriptor buffer p was last read by the round launched two calls ago
    cudaError_t e = cudaEventSynchronize(b->done[p]);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch round wait");
    int tile = 0;
    split_variant_info(b->variant, &tile, nullptr, nullptr);
    plan_round(b, round, tile, *b->h_round[p], true, nullptr, nullptr);
    b->h_round[p]->parity = p;
    lpk_status st = LPK_OK;
    if (b->graph[p] && b->graph_prof[p] != c->profiling) {
        cudaGraphExecDestroy(b->graph[p]);
        cudaGraphDestroy(b->graph_src[p]);
        b->graph[p] = nullptr;
        b->graph_src[p] = nullptr;
    }
    if (!b->graph[p] && (st = build_graph(b, p))) return st;
    cudaEvent_t ea, eb;
    if (b->graph_prof[p] && prof_take(c, ea, eb)) {
        e = cudaGraphExecEventRecordNodeSetEvent(b->graph[p], b->prof_node[p][0], ea);
        if (e == cudaSuccess) e = cudaGraphExecEventRecordNodeSetEvent(b->graph[p], b->prof_node[p][1], eb);
        if (e != cudaSuccess) return cuda_fail(c, e, "profiling event nodes");
    }
    // the output buffers of parity p may still be being copied out (round - 2)
    e = cudaStreamWaitEvent(c->stream, b->copied[p], 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(b->graph[p], c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(b->done[p], c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch graph launch");
    c->launches += 2 + (b->walks.empty() ? 0 : 3);
    b->last_parity = p;
    b->parity ^= 1;
    b->last_round = round;
    return LPK_OK;
}

lpk_status lpk_batch_reset(lpk_batch *b) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    for (auto &w : b->walks) {
        w.totals_done = 0;
        w.g_known = 0;
    }
    return LPK_OK;
}

lpk_status lpk_batch_output(lpk_batch *b, int32_t unit, const lpk_cf32 **d_out) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    if (unit < 0 || unit >= (int32_t)b->units.size()) return fail(b->ctx, LPK_EINVAL, "unit out of range");
    if (!d_out) return fail(b->ctx, LPK_EINVAL, "d_out is NULL");
    *d_out = (const lpk_cf32 *)b->h_units[unit].out[b->last_parity];
    return LPK_OK;
}

lpk_status lpk_batch_copy_out(lpk_batch *b, int32_t unit, lpk_cf32 *host, int64_t cap) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    lpk_ctx *c = b->ctx;
    if (unit < 0 || unit >= (int32_t)b->units.size()) return fail(c, LPK_EINVAL, "unit out of range");
    if (b->last_round < 0) return fail(c, LPK_EINVAL, "no round has run");
    int64_t i0, n;
    unit_extent(b, b->last_round, unit, i0, n);
    if (n > 0 && (!host || cap < n)) return fail(c, LPK_EINVAL, "host buffer is NULL or too small");
    cudaSetDevice(c->device);
    cudaError_t e = n > 0 ? cudaMemcpyAsync(host, b->h_units[unit].out[b->last_parity], sizeof(lpk_cf32) * (size_t)n,
                                            cudaMemcpyDeviceToHost, c->stream)
                          : cudaSuccess;
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "batch output copy");
    return LPK_OK;
}

lpk_status lpk_batch_render(lpk_batch *b, lpk_unit_sink_fn sink, void *user) {
    if (!b || !sink) return fail(b ? b->ctx : nullptr, LPK_EINVAL, "batch or sink is NULL");
    lpk_ctx *c = b->ctx;
    cudaSetDevice(c->device);
    const int nu = (int)b->units.size();
    // staging in the context's pinned pool (kept across batches and calls)
    size_t bytes = 0;
    for (int u = 0; u < nu; ++u) bytes += 2 * (((sizeof(lpk_cf32) * (size_t)b->units[u].round_len) + 255) / 256 * 256);
    lpk_status pst = ensure_pinned(c, bytes);
    if (pst) return pst;
    {
        char *h = (char *)c->h_pinned;
        for (int p = 0; p < 2; ++p) {
            b->staging[p].assign((size_t)nu, nullptr);
            for (int u = 0; u < nu; ++u) {
                b->staging[p][u] = (lpk_cf32 *)h;
                h += ((sizeof(lpk_cf32) * (size_t)b->units[u].round_len) + 255) / 256 * 256;
            }
        }
    }
    std::vector<char> stopped((size_t)nu, 0);
    auto deliver = [&](int64_t round, int p) -> lpk_status {
        cudaError_t e = cudaEventSynchronize(b->copied[p]);
        if (e != cudaSuccess) return cuda_fail(c, e, "output copy wait");
        for (int u = 0; u < nu; ++u) {
            int64_t i0, n;
            unit_extent(b, round, u, i0, n);
            if (n <= 0 || stopped[u]) continue;
            int32_t flow = sink(user, u, b->staging[p][u], n);
            if (flow < 0) return fail(c, LPK_EINVAL, "sink reported an error");
            if (flow == 1) stopped[u] = 1;
        }
        return LPK_OK;
    };
    lpk_status st = LPK_OK;
    for (int64_t r = 0; r < b->n_rounds && !st; ++r) {
        if ((st = lpk_batch_run(b, r))) break;
        const int p = b->last_parity;
        // copies of round r on the copy stream, after the round's graph
        cudaError_t e = cudaStreamWaitEvent(b->copy, b->done[p], 0);
        for (int u = 0; u < nu && e == cudaSuccess; ++u) {
            int64_t i0, n;
            unit_extent(b, r, u, i0, n);
            if (n > 0 && !stopped[u])
                e = cudaMemcpyAsync(b->staging[p][u], b->h_units[u].out[p], sizeof(lpk_cf32) * (size_t)n,
                                    cudaMemcpyDeviceToHost, b->copy);
        }
        if (e == cudaSuccess) e = cudaEventRecord(b->copied[p], b->copy);
        if (e != cudaSuccess) { st = cuda_fail(c, e, "output copy"); break; }
        if (r > 0) st = deliver(r - 1, p ^ 1);  // round r - 1 while round r renders
    }
    if (!st && b->n_rounds > 0) st = deliver(b->n_rounds - 1, b->last_parity);
    cudaStreamSynchronize(b->copy);
    return st;
}

lpk_status lpk_batch_set_config(lpk_batch *b, int32_t variant, int32_t blocks_per_sm) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    return configure(b, variant, blocks_per_sm);
}

lpk_status lpk_batch_get_config(const lpk_batch *b, int32_t *variant, int32_t *bps, int32_t *max_bps) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    if (variant) *variant = b->variant;
    if (bps) *bps = b->bps;
    if (max_bps) *max_bps = b->max_bps;
    return LPK_OK;
}

lpk_status lpk_batch_autotune(lpk_batch *b, int64_t round, int32_t reps, double *ms_table) {
    if (!b) return fail(nullptr, LPK_EINVAL, "batch is NULL");
    lpk_ctx *c = b->ctx;
    if (reps < 1) return fail(c, LPK_EINVAL, "reps must be >= 1");
    if (round < 0 || round >= b->n_rounds) return fail(c, LPK_EINVAL, "round out of range");
    cudaSetDevice(c->device);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    double best = 1e300;
    int best_v = b->variant, best_bps = b->bps;
    lpk_status st = LPK_OK;
    for (int v = 0; v < kSplitVariants && !st; ++v) {
        for (int h = 0; h < 2 && !st; ++h) {
            if (ms_table) ms_table[2 * v + h] = -1.0;
            cudaStreamSynchronize(c->stream);
            if ((st = configure(b, v, 0))) break;
            const int bps = h == 0 ? b->max_bps : b->max_bps / 2;
            if (h == 1 && (bps < 1 || bps == b->max_bps)) continue;
            if ((st = configure(b, v, bps))) break;
            if ((st = lpk_batch_run(b, round))) break;  // warm-up (and graph build)
            cudaEventRecord(t0, c->stream);
            for (int r = 0; r < reps && !st; ++r) st = lpk_batch_run(b, round);
            cudaEventRecord(t1, c->stream);
            if (st) break;
            cudaError_t e = cudaEventSynchronize(t1);
            if (e != cudaSuccess) { st = cuda_fail(c, e, "autotune timing"); break; }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, t0, t1);
            const double per = (double)ms / reps;
            if (ms_table) ms_table[2 * v + h] = per;
            if (per < best) {
                best = per;
                best_v = v;
                best_bps = bps;
            }
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaStreamSynchronize(c->stream);
    if (st) return st;
    return configure(b, best_v, best_bps);
}

}  // extern "C"
