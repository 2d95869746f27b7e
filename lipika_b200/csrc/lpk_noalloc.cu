// lpk_noalloc.cu — a fan-out entry point that allocates no memory.
//
// Some hosts cannot allocate device memory at the point where they render a
// chunk: a real-time SDR emulator thread that must not stall on the CUDA
// allocator, a host that reserved the whole device up front for its own pool,
// or an embedding where only pre-registered buffers may be touched. For them,
// lpk_band_chunk_device_static does what lpk_band_chunk_device does — the
// active list, the per-transmitter occlusion words, the receiver clock walk
// (block totals, group sums, carries, the materialised walk) and, for a
// split-solver band, the anchor records of the chunk's tiles, and the
// flicker points of a clock with a flicker track — in one
// file-scope static device array instead of the context's growable scratch,
// running the same kernels on the same inputs (so the outputs are the same
// bits).
//
// The array lives on every GPU that loads the library until the process exits.
// Every call shares it and it keeps the last call's contents, so each call
// clears what must start at zero; two calls that overlap on the GPU (on any
// stream, from any context on the same device) race on it. Nothing of an
// earlier call is trusted: the walk's block totals and carries are rebuilt
// from master sample 0 on every call, so a call's walk work grows with the
// chunk's master-sample offset (a chunk near the end of a band costs more
// than one near its start).
#include <cmath>
#include <mutex>

#include "lpk_internal.h"

namespace {

constexpr size_t kMaxActive = 256;
constexpr int64_t kMaxWalkBlocks = 1 << 17;      // walk blocks of 4096 master samples (5.4e8 samples)
constexpr int64_t kMaxWalkSpan = 1 << 20;        // master samples one chunk may interpolate over
constexpr size_t kOffActive = 0;
constexpr size_t kOffWords = kOffActive + sizeof(int32_t) * kMaxActive;
constexpr size_t kOffTotals = kOffWords + sizeof(uint32_t) * kMaxActive;
constexpr size_t kOffCarry = kOffTotals + sizeof(double) * kMaxWalkBlocks;
constexpr size_t kOffGsum = kOffCarry + sizeof(double) * (kMaxWalkBlocks + 1);
constexpr size_t kOffEps = (kOffGsum + sizeof(double) * (kMaxWalkBlocks / lpk::kGroupBlocks + 1) + 255) / 256 * 256;
constexpr size_t kOffRecs = (kOffEps + sizeof(double) * kMaxWalkSpan + 255) / 256 * 256;
constexpr size_t kMaxRecsBytes = size_t(32768) * 400;  // split anchor records: 32,768 (tile, transmitter) pairs
                                                       // of 240 + 160 bytes (record + extension)
constexpr size_t kOffFlicker = kOffRecs + kMaxRecsBytes;
constexpr int64_t kMaxFlicker = 8192;             // flicker track points one chunk may read (64 s)
constexpr size_t kStaticBytes = kOffFlicker + sizeof(double) * kMaxFlicker;  // 22.6 MiB

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

std::mutex g_setup_mu;
void *g_static_ptr[64] = {};

// Device address of g_static_scratch on the current device (set up once per
// device, with that device current).
lpk_status static_scratch(lpk_ctx *c, char **out) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (c->device < 0 || c->device >= 64) return lpk::fail(c, LPK_EINVAL, "device index beyond 63");
    if (!g_static_ptr[c->device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return lpk::cuda_fail(c, e, "cudaGetSymbolAddress(static scratch)");
        g_static_ptr[c->device] = p;
    }
    *out = (char *)g_static_ptr[c->device];
    return LPK_OK;
}

}  // namespace

using namespace lpk;

extern "C" lpk_status lpk_band_chunk_device_static(lpk_ctx *c, const lpk_band_desc *band, const int32_t *active,
                                                   int32_t n_active, int64_t i0, int64_t n, const double *d_delta,
                                                   const double *d_rxpos, lpk_cf32 *d_out, uint8_t *d_unocc) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    DevBand b;
    lpk_status st = build_dev_band(c, band, i0, n, b);
    if (st) return st;
    if ((st = check_active(c, active, n_active))) return st;
    if (b.clock_mode == LPK_CLOCK_HOST && n > 0 && !d_delta) return fail(c, LPK_EINVAL, "delta_t is NULL");
    if (b.rx_kind == LPK_RX_PER_SAMPLE && n > 0 && !d_rxpos) return fail(c, LPK_EINVAL, "rx_pos3n is NULL");
    if (n > 0 && !d_out) return fail(c, LPK_EINVAL, "out is NULL");
    b.delta = d_delta;
    b.rxpos = d_rxpos;
    int64_t kA = 0, span = 0, need = 0;
    double sigma = 0.0;
    if (b.clock_mode == LPK_CLOCK_DEVICE_WALK) {
        span = walk_span(band, i0, n, &kA);
        if (span > kMaxWalkSpan)
            return fail(c, LPK_EINVAL, "chunk spans more than 2^20 master-clock samples (static scratch limit); "
                                       "use smaller chunks");
        need = (kA + span - 1) / kWalkBlock;
        if (need + 1 > kMaxWalkBlocks)
            return fail(c, LPK_EINVAL, "chunk lies beyond 2^29 master-clock samples (static scratch limit)");
        sigma = band->clock_allan_1s / std::sqrt(band->clock_master_rate_hz);
    }
    const bool split = use_split(band);
    if (split && split_recs_bytes(c->split_variant, i0, n, n_active) > kMaxRecsBytes)
        return fail(c, LPK_EINVAL, "chunk needs more split anchor records than the static scratch holds "
                                   "(tiles x transmitters > 32768); use smaller chunks");
    cudaSetDevice(c->device);
    char *base = nullptr;
    if ((st = static_scratch(c, &base))) return st;
    int32_t *d_active = (int32_t *)(base + kOffActive);
    uint32_t *d_words = (uint32_t *)(base + kOffWords);
    double *d_tot = (double *)(base + kOffTotals), *d_carry = (double *)(base + kOffCarry);
    double *d_gsum = (double *)(base + kOffGsum);
    double *d_eps = (double *)(base + kOffEps);
    cudaError_t e = cudaMemcpyAsync(d_active, active, sizeof(int32_t) * (size_t)n_active, cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_words, 0, sizeof(uint32_t) * kMaxActive, c->stream);
    if (e == cudaSuccess && span) {
        // The walk's totals and carries are rebuilt from block 0 on every
        // call: nothing of an earlier call is trusted.
        if (need > 0) e = launch_walk_totals(band->clock_seed, sigma, 0, need, d_tot, c->stream);
        if (e == cudaSuccess) e = launch_walk_carries(d_tot, d_gsum, 0, kA / kWalkBlock, need, d_carry, c->stream);
        if (e == cudaSuccess) e = launch_walk_materialize(band->clock_seed, sigma, d_carry, kA, kA + span - 1, d_eps, c->stream);
        b.eps = d_eps;
        b.eps_k0 = kA;
        b.fm = band->clock_master_rate_hz;
    }
    if (e == cudaSuccess && (st = stage_flicker(c, band, i0, n, b, (double *)(base + kOffFlicker), kMaxFlicker)))
        return st;
    if (e == cudaSuccess && split) {  // the split path of lpk_band_chunk_device, on one stream
        b.unocc_words = b.has_antenna ? d_words : nullptr;
        e = launch_band_split(c->split_variant, b, c->d_tx, d_active, n_active, base + kOffRecs, (float2 *)d_out,
                              nullptr, nullptr, nullptr, c->stream);
    } else if (e == cudaSuccess) {
        e = launch_band_reference(b, c->d_tx, d_active, n_active, (float2 *)d_out, d_words, c->stream);
    }
    if (e == cudaSuccess && d_unocc && n_active > 0)
        e = launch_or_flags(d_words, d_unocc, n_active, b.has_antenna ? 0 : (n > 0 ? 1 : 2), c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "static-scratch fan-out");
    return LPK_OK;
}
