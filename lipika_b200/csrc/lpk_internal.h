// lpk_internal.h — context layout shared by the ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/lipika_cuda.h"
#include "lpk_device.cuh"
#include "lpk_walk.cuh"

namespace lpk {

// Cached block totals and group sums of one receiver clock walk (seed,
// master rate, step σ).
struct WalkState {
    uint64_t seed = 0;
    double fm = 0.0, sigma = 0.0;
    int64_t nb_done = 0;   // blocks whose totals are known
    int64_t g_known = 0;   // groups whose sums are stored
    int64_t cap = 0;       // blocks the arrays hold
    double *d_tot = nullptr, *d_carry = nullptr, *d_gsum = nullptr;
};

// Streams, events and pinned round descriptors of a batch (lpk_batch.cu).
// A context keeps the set of the last batch that ended, so the next batch
// skips creating them (pinned allocations and stream creation are slow
// driver calls, and freeing pinned memory synchronises the device).
struct BatchKit {
    void *h_round[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr}, mark[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaStream_t side = nullptr, copy = nullptr;
};
void batch_kit_destroy(BatchKit *k);
}  // namespace lpk

struct lpk_ctx {
    int device = 0;
    std::vector<lpk::WalkState> walks;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // side stream of the chunk entry points: the split path's anchor fits
    // run there, beside the clock walk on `stream`
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
    // scene arena: every table of the uploaded transmitters
    std::vector<void *> scene_allocs;
    std::vector<lpk::DevTx> h_tx;
    lpk::DevTx *d_tx = nullptr;
    int32_t n_tx = 0;
    // growable device scratch for the host-buffer entry points
    void *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    // pinned host staging
    void *h_pinned = nullptr;
    size_t pinned_bytes = 0;
    // measurement hooks
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    size_t prof_used = 0;
    int64_t launches = 0;
    int split_variant = 0;  // launch shape of the split fan-out (LPK_SPLIT_VARIANTS)
    unsigned long long *d_gate_stats = nullptr;  // horizon gate: (stretches tested, skipped)
    // stream-ordered pool for scene tables and batch buffers: kept across
    // scenes and batches, so repeated renders reuse memory without a device
    // synchronisation per allocation
    cudaMemPool_t pool = nullptr;
    lpk::BatchKit *batch_kit = nullptr;  // kept from the last batch (see BatchKit)
};

namespace lpk {

lpk_status fail(lpk_ctx *ctx, lpk_status code, const std::string &msg);
lpk_status cuda_fail(lpk_ctx *ctx, cudaError_t e, const char *what);
lpk_status ensure_scratch(lpk_ctx *ctx, size_t bytes);
lpk_status ensure_pinned(lpk_ctx *ctx, size_t bytes);
// Allocate / free from the context's pool, ordered on its stream.
cudaError_t pool_alloc(lpk_ctx *ctx, void **p, size_t bytes);
void pool_free(lpk_ctx *ctx, void *p);
lpk_status build_dev_band(lpk_ctx *ctx, const lpk_band_desc *b, int64_t i0, int64_t n, DevBand &out);
lpk_status check_active(lpk_ctx *ctx, const int32_t *active, int32_t n_active);

// launchers (lpk_kernels.cu)
cudaError_t launch_band_reference(const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                                  int32_t n_active, float2 *d_out, uint32_t *d_unocc, cudaStream_t s);
// The tuned all-FP64 fan-out (LPK_SOLVER_FP64_TUNED).
cudaError_t launch_band_fp64(const DevBand &b, const DevTx *d_tx, const int32_t *d_active, int32_t n_active,
                             float2 *d_out, uint32_t *d_unocc, cudaStream_t s);
cudaError_t launch_tx_contribution(const DevBand &b, const DevTx *d_tx, int32_t tx, float2 *d_out,
                                   double *d_phase, double *d_temit, double *d_range, cudaStream_t s);
cudaError_t launch_rx_chain(const DevBand &b, float2 *d_iq, cudaStream_t s);
cudaError_t launch_band_delta(const DevBand &b, double *d_out, cudaStream_t s);
cudaError_t launch_sample_times(double fs, int64_t i0, int64_t n, double *d_out, cudaStream_t s);
// Split-precision fan-out (anchor kernel + per-sample kernel) in launch
// shape `variant`; d_recs holds split_recs_bytes(variant, i0, n, n_active)
// bytes. The dbg arrays (single transmitter only, may be NULL) receive the
// reduced phase, emission time and delay.
bool split_variant_info(int variant, int *tile, int *threads, int *min_blocks);
size_t split_recs_bytes(int variant, int64_t i0, int64_t n, int32_t n_active);
// The two halves of launch_band_split: the anchor fits (into d_recs) and
// the fan-out that reads them.
cudaError_t launch_split_anchor(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                               int32_t n_active, void *d_recs, cudaStream_t s);
cudaError_t launch_split_fanout(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                                int32_t n_active, void *d_recs, float2 *d_out, double *dbg_phase, double *dbg_temit,
                                double *dbg_delay, cudaStream_t s);
cudaError_t launch_band_split(int variant, const DevBand &b, const DevTx *d_tx, const int32_t *d_active,
                              int32_t n_active, void *d_recs, float2 *d_out, double *dbg_phase, double *dbg_temit,
                              double *dbg_delay, cudaStream_t s);
// True when the band can take the split path (stationary receiver).
inline bool use_split(const lpk_band_desc *d) {
    return d->solver == LPK_SOLVER_SPLIT && (d->rx_kind == LPK_RX_STATIONARY || d->rx_kind == LPK_RX_KEPLER);
}
cudaError_t launch_or_flags(const uint32_t *d_uw, uint8_t *d_unocc, int32_t n_active, int mode, cudaStream_t s);
// Totals of scan blocks [b_from, b_to).
cudaError_t launch_walk_totals(uint64_t seed, double sigma, int64_t b_from, int64_t b_to, double *d_tot,
                               cudaStream_t s);
// carry(b) for b in [bA, bB] (totals below bB known; sums of groups below
// g_known stored in d_gsum; afterwards those below bB / kGroupBlocks are).
cudaError_t launch_walk_carries(const double *d_tot, double *d_gsum, int64_t g_known, int64_t bA, int64_t bB,
                                double *d_carry, cudaStream_t s);
cudaError_t launch_walk_materialize(uint64_t seed, double sigma, const double *d_carry, int64_t kA, int64_t kB,
                                    double *d_eps, cudaStream_t s);
// Device walk for a band chunk: ensure carries, materialise ε over the
// chunk's master range into `eps_region` of the scratch (lpk_abi.cu).
lpk_status prepare_walk(lpk_ctx *ctx, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, double *d_eps,
                        int64_t eps_cap);
int64_t walk_span(const lpk_band_desc *d, int64_t i0, int64_t n, int64_t *kA);
// The device constants of a circular Keplerian orbit (lpk_traj.cu).
bool make_orbit(const lpk_kepler_orbit &k, DevOrbit &o);
// Device-clock inputs of a band chunk in one scratch region: the walk
// values (DEVICE_WALK) followed by the staged flicker points (a flicker
// track). clock_region_bytes: the region's size (256-byte aligned parts);
// prepare_clock fills it and points b at it (lpk_abi.cu).
size_t clock_region_bytes(const lpk_band_desc *d, int64_t i0, int64_t n);
lpk_status prepare_clock(lpk_ctx *ctx, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, char *region);
// The flicker points of a chunk copied to dst (at most cap) and b pointed
// at them; nothing without a flicker track.
lpk_status stage_flicker(lpk_ctx *ctx, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, double *dst,
                         int64_t cap);
// Record a profiling event pair around a fan-out launch (no-op when off).
void prof_begin(lpk_ctx *ctx);
void prof_end(lpk_ctx *ctx);
// Take the next profiling event pair for a fan-out that is timed by event
// nodes inside a graph (false when profiling is off).
bool prof_take(lpk_ctx *ctx, cudaEvent_t &a, cudaEvent_t &b);
cudaError_t launch_fp64_probe(double *d_out, int blocks, int iters, cudaStream_t s);
cudaError_t launch_solve(const DevTx *d_tx, int32_t tx, const double *d_obs, const double *d_t, int64_t n,
                         double epoch, int32_t iterations, double inv_c, double *d_temit, double *d_range,
                         cudaStream_t s);

}  // namespace lpk
