// lpk_abi.cu — context, transmitter upload and the kernel-level C ABI
// (include/lipika_cuda.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lpk_internal.h"

using lpk::DevBand;
using lpk::DevTx;

namespace {
std::mutex g_err_mu;
std::string g_err;
}  // namespace

namespace lpk {

lpk_status fail(lpk_ctx *ctx, lpk_status code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
    return code;
}

lpk_status cuda_fail(lpk_ctx *ctx, cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return fail(ctx, LPK_ECUDA, buf);
}

lpk_status ensure_scratch(lpk_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->scratch_bytes) return LPK_OK;
    if (ctx->d_scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_scratch);
        ctx->d_scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(&ctx->d_scratch, want);
    if (e != cudaSuccess) {
        ctx->d_scratch = nullptr;
        return fail(ctx, LPK_ENOMEM, std::string("device scratch allocation failed: ") + cudaGetErrorString(e));
    }
    ctx->scratch_bytes = want;
    return LPK_OK;
}

lpk_status ensure_pinned(lpk_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->pinned_bytes) return LPK_OK;
    if (ctx->h_pinned) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->h_pinned);
        ctx->h_pinned = nullptr;
        ctx->pinned_bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMallocHost(&ctx->h_pinned, want);
    if (e != cudaSuccess) {
        ctx->h_pinned = nullptr;
        return fail(ctx, LPK_ENOMEM, std::string("pinned staging allocation failed: ") + cudaGetErrorString(e));
    }
    ctx->pinned_bytes = want;
    return LPK_OK;
}

cudaError_t pool_alloc(lpk_ctx *ctx, void **p, size_t bytes) {
    return cudaMallocFromPoolAsync(p, bytes ? bytes : 16, ctx->pool, ctx->stream);
}

void pool_free(lpk_ctx *ctx, void *p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}

static bool finite(double x) { return std::isfinite(x); }

// Lower an lpk_band_desc to the device constants, computing once what the
// reference computes once per band (generate_band, pipeline.rs:853-895;
// RxChain::from_config and PostOp parameters, rx/mod.rs:83-137).
lpk_status build_dev_band(lpk_ctx *ctx, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b) {
    memset(&b, 0, sizeof b);
    if (!d) return fail(ctx, LPK_EINVAL, "band descriptor is NULL");
    if (!(d->fs_hz > 0.0) || !finite(d->fs_hz)) return fail(ctx, LPK_EINVAL, "band fs_hz must be positive and finite");
    if (!finite(d->lo_hz) || !finite(d->epoch_unix)) return fail(ctx, LPK_EINVAL, "band lo_hz/epoch must be finite");
    if (!(d->noise_power_w >= 0.0) && !(d->noise_power_w < 0.0))
        return fail(ctx, LPK_EINVAL, "band noise_power_w is NaN");
    if (n < 0 || i0 < 0) return fail(ctx, LPK_EINVAL, "chunk start and length must be non-negative");
    if (d->rx_kind != LPK_RX_STATIONARY && d->rx_kind != LPK_RX_PER_SAMPLE && d->rx_kind != LPK_RX_KEPLER)
        return fail(ctx, LPK_EINVAL, "unknown rx_kind");
    if (d->rx_kind == LPK_RX_KEPLER) {
        if (!make_orbit(d->rx_orbit, b.rx_orb)) return fail(ctx, LPK_EINVAL, "bad receiver orbit");
        // fl(epoch + tu) - orbit epoch is exact (Sterbenz) when the orbit
        // epoch is 0 or within a factor of two of every query time; then the
        // split path's smooth receiver model plus the query's rounding offset
        // is the reference's orbit time
        const double e0 = d->rx_orbit.epoch_unix, ep = d->epoch_unix;
        b.rx_de = ep - e0;
        b.rx_split_ok = e0 == 0.0 || (ep > 0.0 && e0 >= 0.6 * ep && e0 <= 1.6 * ep);
    }
    if (d->clock_mode != LPK_CLOCK_HOST && d->clock_mode != LPK_CLOCK_DETERMINISTIC &&
        d->clock_mode != LPK_CLOCK_DEVICE_WALK)
        return fail(ctx, LPK_EINVAL, "unknown clock_mode");
    if (d->clock_mode == LPK_CLOCK_DEVICE_WALK &&
        (!(d->clock_master_rate_hz > 0.0) || !finite(d->clock_master_rate_hz) || !(d->clock_allan_1s >= 0.0) ||
         !finite(d->clock_allan_1s)))
        return fail(ctx, LPK_EINVAL, "device clock walk needs a positive master rate and allan >= 0");
    if (d->flicker_delta_s && d->clock_mode != LPK_CLOCK_HOST && d->flicker_n < 2)
        return fail(ctx, LPK_EINVAL, "flicker track needs at least two points");
    if (d->n_post < 0 || d->n_post > 3) return fail(ctx, LPK_EINVAL, "n_post must be 0..3");
    if (d->solver != LPK_SOLVER_REFERENCE && d->solver != LPK_SOLVER_SPLIT && d->solver != LPK_SOLVER_FP64_TUNED)
        return fail(ctx, LPK_EINVAL, "unknown solver");
    b.epoch = d->epoch_unix;
    b.fs = d->fs_hz;
    b.lo = d->lo_hz;
    b.inv_c = 1.0 / kSpeedOfLight;
    b.i0 = i0;
    b.n = n;
    b.rx_kind = d->rx_kind;
    b.clock_mode = d->clock_mode;
    for (int k = 0; k < 3; ++k) b.rx[k] = d->rx_ecef[k];
    b.clock_offset = d->clock_offset_s;
    b.clock_y0 = d->clock_y0;
    if (d->noise_power_w > 0.0) {
        b.has_noise = 1;
        b.noise_std = (float)std::sqrt(d->noise_power_w / 2.0);  // channel/mod.rs:328
        b.noise_seed = d->noise_seed;
    }
    b.has_antenna = d->has_antenna;
    b.has_cutoff = d->has_cutoff;
    b.ant_peak = d->ant_peak_dbi;
    b.ant_horizon = d->ant_horizon_dbi;
    b.ant_fb = d->ant_fb_db;
    b.ant_cutoff = d->ant_cutoff_deg;
    b.n_post = d->n_post;
    b.gate_stats = ctx ? ctx->d_gate_stats : nullptr;
    for (int k = 0; k < d->n_post; ++k) {
        const lpk_post_op &op = d->post[k];
        b.post_kind[k] = op.kind;
        if (op.kind == LPK_POST_GAIN) {
            b.post_a[k] = powf(10.0f, (float)(op.param / 20.0));
        } else if (op.kind == LPK_POST_NONLINEARITY) {
            if (!(op.param > 0.0)) return fail(ctx, LPK_EINVAL, "nonlinearity iip3_w must be positive");
            b.post_a[k] = (float)(4.0 / 3.0 / op.param);
        } else if (op.kind == LPK_POST_ADC) {
            uint32_t bits = op.bits < 2 ? 2 : op.bits;
            if (bits > 63) return fail(ctx, LPK_EINVAL, "adc bits must be at most 63");
            float fs = (float)op.param;
            float levels = (float)((1ULL << (bits - 1)) - 1ULL);
            b.post_a[k] = fs;
            b.post_b[k] = fs / levels;
        } else {
            return fail(ctx, LPK_EINVAL, "unknown post op kind");
        }
    }
    return LPK_OK;
}

// Master-grid indices [kA, kA + span) the chunk's Δt interpolation reads
// (one index of margin on each side of what ClockStream::delta_t_at uses).
int64_t walk_span(const lpk_band_desc *d, int64_t i0, int64_t n, int64_t *kA_out) {
    const double fs = d->fs_hz, fm = d->clock_master_rate_hz;
    double x0 = ((double)i0 / fs) * fm;
    double x1 = ((double)(i0 + (n > 0 ? n - 1 : 0)) / fs) * fm;
    int64_t kA = x0 <= 0.0 ? 0 : (int64_t)std::floor(x0);
    int64_t kB = (x1 <= 0.0 ? 0 : (int64_t)std::floor(x1)) + 2;
    kA = kA > 0 ? kA - 1 : 0;
    *kA_out = kA;
    return kB - kA + 1;
}

lpk_status prepare_walk(lpk_ctx *c, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, double *d_eps,
                        int64_t eps_cap) {
    int64_t kA;
    int64_t span = walk_span(d, i0, n, &kA);
    if (span > eps_cap) return fail(c, LPK_EINVAL, "walk span exceeds its scratch region");
    const int64_t kB = kA + span - 1;
    const double sigma = d->clock_allan_1s / std::sqrt(d->clock_master_rate_hz);  // clock/mod.rs:275
    WalkState *w = nullptr;
    for (auto &s : c->walks)
        if (s.seed == d->clock_seed && s.fm == d->clock_master_rate_hz && s.sigma == sigma) w = &s;
    if (!w) {
        c->walks.push_back(WalkState{});
        w = &c->walks.back();
        w->seed = d->clock_seed;
        w->fm = d->clock_master_rate_hz;
        w->sigma = sigma;
    }
    const int64_t bA = kA / kWalkBlock, need = kB / kWalkBlock;  // carries of blocks [bA, need]
    if (need + 1 > w->cap) {
        int64_t cap = w->cap ? w->cap : 1024;
        while (cap < need + 1) cap *= 2;
        double *tot = nullptr, *car = nullptr, *gs = nullptr;
        cudaError_t e = cudaMalloc(&tot, sizeof(double) * (size_t)cap);
        if (e == cudaSuccess) e = cudaMalloc(&car, sizeof(double) * (size_t)(cap + 1));
        if (e == cudaSuccess) e = cudaMalloc(&gs, sizeof(double) * (size_t)(cap / kGroupBlocks + 1));
        if (e != cudaSuccess) {
            if (tot) cudaFree(tot);
            if (car) cudaFree(car);
            return fail(c, LPK_ENOMEM, "clock walk carry allocation failed");
        }
        if (w->nb_done > 0)
            cudaMemcpyAsync(tot, w->d_tot, sizeof(double) * (size_t)w->nb_done, cudaMemcpyDeviceToDevice, c->stream);
        if (w->g_known > 0)
            cudaMemcpyAsync(gs, w->d_gsum, sizeof(double) * (size_t)w->g_known, cudaMemcpyDeviceToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
        if (w->d_tot) cudaFree(w->d_tot);
        if (w->d_carry) cudaFree(w->d_carry);
        if (w->d_gsum) cudaFree(w->d_gsum);
        w->d_tot = tot;
        w->d_carry = car;
        w->d_gsum = gs;
        w->cap = cap;
    }
    cudaError_t e = cudaSuccess;
    if (need > w->nb_done) {
        e = launch_walk_totals(w->seed, w->sigma, w->nb_done, need, w->d_tot, c->stream);
        c->launches += 1;
        if (e != cudaSuccess) return cuda_fail(c, e, "clock walk totals");
        w->nb_done = need;
    }
    e = launch_walk_carries(w->d_tot, w->d_gsum, w->g_known, bA, need, w->d_carry, c->stream);
    c->launches += 1;
    if (e != cudaSuccess) return cuda_fail(c, e, "clock walk carries");
    if (need / kGroupBlocks > w->g_known) w->g_known = need / kGroupBlocks;
    e = launch_walk_materialize(w->seed, w->sigma, w->d_carry, kA, kB, d_eps, c->stream);
    c->launches += 1;
    if (e != cudaSuccess) return cuda_fail(c, e, "clock walk materialisation");
    b.eps = d_eps;
    b.eps_k0 = kA;
    b.fm = d->clock_master_rate_hz;
    return LPK_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Coarse flicker points [m_lo, m_lo + count) that band samples [i0, i0 + n)
// read (band_flicker: points floor(t·128) and floor(t·128) + 1), with one
// point of margin on either side, clamped to the track; -1 when the track
// does not reach the chunk's last sample.
static int64_t flicker_span(const lpk_band_desc *d, int64_t i0, int64_t n, int64_t *m_lo) {
    const double fs = d->fs_hz;
    const double x0 = ((double)i0 / fs) * kFlickerRate;
    const double x1 = ((double)(i0 + (n > 0 ? n - 1 : 0)) / fs) * kFlickerRate;
    const int64_t a = x0 <= 0.0 ? 0 : (int64_t)std::floor(x0);
    const int64_t need = (x1 <= 0.0 ? 0 : (int64_t)std::floor(x1)) + 1;
    if (need >= d->flicker_n) return -1;
    const int64_t lo = a > 0 ? a - 1 : 0, hi = need + 1 < d->flicker_n ? need + 1 : need;
    *m_lo = lo;
    return hi - lo + 1;
}

static bool uses_flicker(const lpk_band_desc *d) {
    return d->flicker_delta_s && d->clock_mode != LPK_CLOCK_HOST;
}

size_t clock_region_bytes(const lpk_band_desc *d, int64_t i0, int64_t n) {
    size_t bytes = 0;
    int64_t k = 0;
    if (d->clock_mode == LPK_CLOCK_DEVICE_WALK) bytes += align256(sizeof(double) * (size_t)walk_span(d, i0, n, &k));
    if (uses_flicker(d)) {
        const int64_t cnt = flicker_span(d, i0, n, &k);  // -1 (a short track): prepare_clock refuses it
        bytes += align256(sizeof(double) * (size_t)(cnt > 0 ? cnt : 1));
    }
    return bytes;
}

lpk_status prepare_clock(lpk_ctx *c, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, char *region) {
    size_t off = 0;
    int64_t k = 0;
    if (d->clock_mode == LPK_CLOCK_DEVICE_WALK) {
        const int64_t span = walk_span(d, i0, n, &k);
        lpk_status st = prepare_walk(c, d, i0, n, b, (double *)region, span);
        if (st) return st;
        off = align256(sizeof(double) * (size_t)span);
    }
    return stage_flicker(c, d, i0, n, b, (double *)(region + off), INT64_MAX);
}

lpk_status stage_flicker(lpk_ctx *c, const lpk_band_desc *d, int64_t i0, int64_t n, DevBand &b, double *dst,
                         int64_t cap) {
    if (!uses_flicker(d)) return LPK_OK;
    int64_t m_lo = 0;
    const int64_t cnt = flicker_span(d, i0, n, &m_lo);
    if (cnt < 2) return fail(c, LPK_EINVAL, "flicker track shorter than the chunk");
    if (cnt > cap) return fail(c, LPK_EINVAL, "chunk spans more flicker points than its scratch holds");
    cudaError_t e = cudaMemcpyAsync(dst, d->flicker_delta_s + m_lo, sizeof(double) * (size_t)cnt,
                                    cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "flicker track upload");
    b.flicker = dst;
    b.flicker_m0 = m_lo;
    b.flicker_n = cnt;
    return LPK_OK;
}

void prof_begin(lpk_ctx *c) {
    if (!c->profiling) return;
    if (c->prof_used == c->prof_events.size()) {
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess) return;
        if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return; }
        c->prof_events.push_back({a, b});
    }
    cudaEventRecord(c->prof_events[c->prof_used].first, c->stream);
}

bool prof_take(lpk_ctx *c, cudaEvent_t &a, cudaEvent_t &b) {
    if (!c->profiling) return false;
    if (c->prof_used == c->prof_events.size()) {
        cudaEvent_t x, y;
        if (cudaEventCreate(&x) != cudaSuccess) return false;
        if (cudaEventCreate(&y) != cudaSuccess) { cudaEventDestroy(x); return false; }
        c->prof_events.push_back({x, y});
    }
    a = c->prof_events[c->prof_used].first;
    b = c->prof_events[c->prof_used].second;
    ++c->prof_used;
    return true;
}

void prof_end(lpk_ctx *c) {
    if (!c->profiling || c->prof_used >= c->prof_events.size()) return;
    cudaEventRecord(c->prof_events[c->prof_used].second, c->stream);
    ++c->prof_used;
}

lpk_status check_active(lpk_ctx *ctx, const int32_t *active, int32_t n_active) {
    if (n_active < 0 || n_active > 256) return fail(ctx, LPK_EINVAL, "n_active must be 0..256");
    if (n_active > 0 && !active) return fail(ctx, LPK_EINVAL, "active_tx is NULL");
    for (int32_t k = 0; k < n_active; ++k)
        if (active[k] < 0 || active[k] >= ctx->n_tx)
            return fail(ctx, LPK_EINVAL, "active_tx index out of range of the uploaded scene");
    return LPK_OK;
}

}  // namespace lpk

using namespace lpk;

extern "C" {

const char *lpk_version(void) { return "lipika_b200 0.1 (sm_100a)"; }

const char *lpk_global_last_error(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    static thread_local std::string copy;
    copy = g_err;
    return copy.c_str();
}

const char *lpk_last_error(const lpk_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

void *lpk_ctx_stream(lpk_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

lpk_status lpk_profile_enable(lpk_ctx *c, int32_t on) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    c->profiling = on != 0;
    return LPK_OK;
}

lpk_status lpk_profile_reset(lpk_ctx *c) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    cudaStreamSynchronize(c->stream);
    c->prof_used = 0;
    c->launches = 0;
    return LPK_OK;
}

lpk_status lpk_profile_read(lpk_ctx *c, double *ms, int64_t *fan, int64_t *all) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "profile synchronize");
    double total = 0.0;
    for (size_t i = 0; i < c->prof_used; ++i) {
        float t = 0.0f;
        e = cudaEventElapsedTime(&t, c->prof_events[i].first, c->prof_events[i].second);
        if (e != cudaSuccess) return cuda_fail(c, e, "profile event");
        total += t;
    }
    if (ms) *ms = total;
    if (fan) *fan = (int64_t)c->prof_used;
    if (all) *all = c->launches;
    return LPK_OK;
}

lpk_status lpk_gate_stats(lpk_ctx *c, int64_t *tested, int64_t *skipped, int32_t reset) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    cudaSetDevice(c->device);
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(h, c->d_gate_stats, sizeof h, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) e = cudaMemset(c->d_gate_stats, 0, sizeof h);
    if (e != cudaSuccess) return cuda_fail(c, e, "gate statistics");
    if (tested) *tested = (int64_t)h[0];
    if (skipped) *skipped = (int64_t)h[1];
    return LPK_OK;
}

lpk_status lpk_probe_fp64_peak(lpk_ctx *c, double *tflops) {
    if (!c || !tflops) return fail(c, LPK_EINVAL, "NULL argument");
    cudaSetDevice(c->device);
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "device properties");
    const int blocks = prop.multiProcessorCount * 8, iters = 1 << 14;
    lpk_status st = ensure_scratch(c, sizeof(double) * 256 * (size_t)blocks);
    if (st) return st;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        e = cudaEventRecord(c->ev_start, c->stream);
        if (e == cudaSuccess) e = launch_fp64_probe((double *)c->d_scratch, blocks, iters, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_stop, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(c->ev_stop);
        float t = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, c->ev_start, c->ev_stop);
        if (e != cudaSuccess) return cuda_fail(c, e, "fp64 probe");
        double flops = 2.0 * 8.0 * (double)iters * 256.0 * (double)blocks;
        if (rep > 0 && t > 0.0f) best = std::fmax(best, flops / (t * 1e-3) / 1e12);
    }
    *tflops = best;
    return LPK_OK;
}

lpk_status lpk_ctx_create(lpk_ctx **out, int32_t device) {
    if (!out) return fail(nullptr, LPK_EINVAL, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) return fail(nullptr, LPK_EINVAL, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    lpk_ctx *c = new (std::nothrow) lpk_ctx();
    if (!c) return fail(nullptr, LPK_ENOMEM, "context allocation failed");
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev_stop);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&c->pool, &props);
        uint64_t keep = ~0ull;  // never trim: memory returns to this pool, not to the driver
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_gate_stats, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(c->d_gate_stats, 0, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        lpk_status st = cuda_fail(nullptr, e, "stream/event creation");
        lpk_ctx_destroy(c);
        return st;
    }
    *out = c;
    return LPK_OK;
}

static void free_scene(lpk_ctx *c) {
    for (void *p : c->scene_allocs) pool_free(c, p);
    c->scene_allocs.clear();
    c->h_tx.clear();
    c->d_tx = nullptr;
    c->n_tx = 0;
}

void lpk_ctx_destroy(lpk_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_scene(c);
    if (c->batch_kit) lpk::batch_kit_destroy(c->batch_kit);
    for (auto &w : c->walks) {
        if (w.d_tot) cudaFree(w.d_tot);
        if (w.d_carry) cudaFree(w.d_carry);
        if (w.d_gsum) cudaFree(w.d_gsum);
    }
    for (auto &p : c->prof_events) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    if (c->d_scratch) cudaFree(c->d_scratch);
    if (c->d_gate_stats) cudaFree(c->d_gate_stats);
    if (c->pool) {
        cudaStreamSynchronize(c->stream);
        cudaMemPoolDestroy(c->pool);
    }
    if (c->h_pinned) cudaFreeHost(c->h_pinned);
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->ev_stop) cudaEventDestroy(c->ev_stop);
    if (c->aux) cudaStreamSynchronize(c->aux);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->aux) cudaStreamDestroy(c->aux);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static lpk_status upload_bytes(lpk_ctx *c, const void *src, size_t bytes, void **dst) {
    *dst = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = pool_alloc(c, dst, bytes);
    if (e != cudaSuccess) return fail(c, LPK_ENOMEM, std::string("scene allocation failed: ") + cudaGetErrorString(e));
    c->scene_allocs.push_back(*dst);
    // pageable source: the copy has consumed it when the call returns
    e = src ? cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, c->stream)
            : cudaMemsetAsync(*dst, 0, bytes, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "scene upload");
    return LPK_OK;
}

lpk_status lpk_scene_upload(lpk_ctx *c, const lpk_tx_desc *tx, int32_t n_tx) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (n_tx < 0 || (n_tx > 0 && !tx)) return fail(c, LPK_EINVAL, "bad transmitter array");
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_scene(c);
    std::vector<DevTx> h((size_t)n_tx);
    for (int32_t i = 0; i < n_tx; ++i) {
        const lpk_tx_desc &s = tx[i];
        DevTx &d = h[i];
        memset(&d, 0, sizeof d);
        if (!(s.carrier_hz > 0.0) || !std::isfinite(s.carrier_hz))
            return fail(c, LPK_EINVAL, "transmitter carrier_hz must be positive and finite");
        if (!(s.tx_power_w >= 0.0) || !std::isfinite(s.tx_power_w))
            return fail(c, LPK_EINVAL, "transmitter tx_power_w must be finite and non-negative");
        d.traj_kind = s.traj_kind;
        d.sig_kind = s.sig_kind;
        d.nav_kind = s.nav_kind;
        d.has_repeat = s.has_repeat;
        d.sx = s.stationary_ecef[0];
        d.sy = s.stationary_ecef[1];
        d.sz = s.stationary_ecef[2];
        if (s.traj_kind == LPK_TX_TRAJ_PRECOMPUTED) {
            if (s.grid_n < 2 || !s.grid_xyz || !(s.grid_dt_s > 0.0))
                return fail(c, LPK_EINVAL, "precomputed trajectory needs >= 2 grid points and dt > 0");
            std::vector<double4> g((size_t)s.grid_n);
            for (int64_t k = 0; k < s.grid_n; ++k)
                g[k] = make_double4(s.grid_xyz[k], s.grid_xyz[s.grid_n + k], s.grid_xyz[2 * s.grid_n + k], 0.0);
            void *p;
            lpk_status st = upload_bytes(c, g.data(), sizeof(double4) * g.size(), &p);
            if (st) return st;
            d.grid = (const double4 *)p;
            d.grid_n = s.grid_n;
            {  // path_bounds, src/geometry/precomputed.rs:88-107 (the horizon gate's bounds)
                double max_seg2 = 0.0, max_r2 = 0.0;
                bool finite_all = true;
                for (int64_t k = 0; k < s.grid_n; ++k) {
                    const double4 q = g[k];
                    const double r2 = q.x * q.x + q.y * q.y + q.z * q.z;
                    finite_all &= std::isfinite(r2);
                    if (r2 > max_r2) max_r2 = r2;
                    if (k + 1 < s.grid_n) {
                        const double ex = g[k + 1].x - q.x, ey = g[k + 1].y - q.y, ez = g[k + 1].z - q.z;
                        const double seg2 = ex * ex + ey * ey + ez * ez;
                        finite_all &= std::isfinite(seg2);
                        if (seg2 > max_seg2) max_seg2 = seg2;
                    }
                }
                d.max_speed = finite_all ? std::sqrt(max_seg2) / s.grid_dt_s : std::nan("");
                d.max_radius = finite_all ? std::sqrt(max_r2) : std::nan("");
            }
            d.t0 = s.grid_t0_unix;
            d.dt = s.grid_dt_s;
            d.inv_dt = 1.0 / s.grid_dt_s;
        } else if (s.traj_kind != LPK_TX_TRAJ_STATIONARY) {
            return fail(c, LPK_EINVAL, "unknown trajectory kind");
        }
        d.carrier = s.carrier_hz;
        d.neg_tau_src = -kTau * s.carrier_hz;                              // channel/mod.rs:239
        double wavelength = kSpeedOfLight / s.carrier_hz;                 // :209
        d.amp_factor = (wavelength / (2.0 * kTau)) * std::sqrt(s.tx_power_w);  // :210, :243
        d.epoch_rel = s.epoch_rel_s;
        d.rate = s.rate_hz;
        d.repeat_from = s.repeat_from;
        d.n_sym = s.n_sym;
        void *p = nullptr;
        lpk_status st = LPK_OK;
        switch (s.sig_kind) {
        case LPK_SIG_CW:
            d.cw_omega = kTau * s.cw_offset_hz;  // cw.rs:43
            d.cw_phase0 = s.cw_phase0;
            d.cw_anchored = s.cw_anchored;
            break;
        case LPK_SIG_BPSK:
            if (s.n_sym < 0 || (s.n_sym > 0 && !s.pm_bits)) return fail(c, LPK_EINVAL, "bpsk table missing");
            st = upload_bytes(c, s.pm_bits, (size_t)s.n_sym, &p);
            d.pm = (const int8_t *)p;
            break;
        case LPK_SIG_OOK:
            if (s.n_sym < 0 || (s.n_sym > 0 && !s.ook_bits)) return fail(c, LPK_EINVAL, "ook table missing");
            st = upload_bytes(c, s.ook_bits, (size_t)s.n_sym, &p);
            d.ook = (const uint8_t *)p;
            break;
        case LPK_SIG_QAM16:
            if (s.n_sym < 0 || (s.n_sym > 0 && !s.symbols)) return fail(c, LPK_EINVAL, "qam16 table missing");
            st = upload_bytes(c, s.symbols, sizeof(float2) * (size_t)s.n_sym, &p);
            d.sym = (const float2 *)p;
            break;
        case LPK_SIG_CA_CODE:
            if (!s.chips) return fail(c, LPK_EINVAL, "ca_code chip table missing");
            for (int k = 0; k < 1023; ++k) {
                if (s.chips[k] != 1 && s.chips[k] != -1) return fail(c, LPK_EINVAL, "ca_code chips must be ±1");
                if (s.chips[k] < 0) d.chip_neg[k >> 5] |= 1u << (k & 31);
            }
            d.nav_seed = s.nav_seed;
            if (s.nav_kind == LPK_NAV_FULL) {
                if (s.nav_n < 0 || (s.nav_n > 0 && !s.nav_bits)) return fail(c, LPK_EINVAL, "nav table missing");
                st = upload_bytes(c, s.nav_bits, (size_t)s.nav_n, &p);
                d.nav_bits = (const int8_t *)p;
                d.nav_n = s.nav_n;
            } else if (s.nav_kind != LPK_NAV_OFF && s.nav_kind != LPK_NAV_DUMMY) {
                return fail(c, LPK_EINVAL, "unknown nav kind");
            }
            break;
        default:
            return fail(c, LPK_EINVAL, "unknown signal kind");
        }
        if (st) return st;
        if ((s.sig_kind == LPK_SIG_BPSK || s.sig_kind == LPK_SIG_OOK || s.sig_kind == LPK_SIG_QAM16) &&
            !(s.rate_hz > 0.0))
            return fail(c, LPK_EINVAL, "symbol rate must be positive");
        if (s.has_gate) {
            if (!(s.gate_period_s > 0.0) || !std::isfinite(s.gate_period_s) || s.gate_n < 0 ||
                (s.gate_n > 0 && !s.gate_on))
                return fail(c, LPK_EINVAL, "bad burst gate");
            d.has_gate = 1;
            d.gate_n = s.gate_n;
            d.gate_period = s.gate_period_s;
            d.gate_phase = s.gate_phase_s;
            st = upload_bytes(c, s.gate_on, sizeof(double2) * (size_t)s.gate_n, &p);
            if (st) return st;
            d.gate_on = (const double2 *)p;
        }
    }
    void *p;
    lpk_status st = upload_bytes(c, h.data(), sizeof(DevTx) * h.size(), &p);
    if (st) return st;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "scene upload");
    c->d_tx = (DevTx *)p;
    c->h_tx = std::move(h);
    c->n_tx = n_tx;
    return LPK_OK;
}

// Split path of a chunk entry point: the anchor fits on the side stream
// (after everything already queued on the context's stream, so the previous
// chunk's fan-out has read its records), the walk on the main stream, then
// the fan-out once both are done.
static cudaError_t split_fork_anchor(lpk_ctx *c, const DevBand &b, const int32_t *d_active, int32_t n_active,
                                     void *d_recs) {
    cudaError_t e = cudaEventRecord(c->ev_fork, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->aux, c->ev_fork, 0);
    if (e == cudaSuccess) e = launch_split_anchor(c->split_variant, b, c->d_tx, d_active, n_active, d_recs, c->aux);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_join, c->aux);
    return e;
}

lpk_status lpk_band_chunk_device(lpk_ctx *c, const lpk_band_desc *band, const int32_t *active,
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
    cudaSetDevice(c->device);
    // active list, unoccluded words and the clock walk live in the scratch
    size_t off_uw = align256(sizeof(int32_t) * 256);
    size_t off_eps = off_uw + align256(sizeof(uint32_t) * 256);
    const size_t clk_bytes = clock_region_bytes(band, i0, n);
    const bool split = use_split(band);
    size_t off_recs = off_eps + clk_bytes;
    size_t recs = split ? align256(split_recs_bytes(c->split_variant, i0, n, n_active)) : 0;
    if ((st = ensure_scratch(c, off_recs + recs))) return st;
    int32_t *d_active = (int32_t *)c->d_scratch;
    uint32_t *d_uw = (uint32_t *)((char *)c->d_scratch + off_uw);
    cudaError_t e = cudaMemcpyAsync(d_active, active, sizeof(int32_t) * (size_t)n_active, cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_uw, 0, sizeof(uint32_t) * 256, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "chunk setup");
    if (split && (e = split_fork_anchor(c, b, d_active, n_active, (char *)c->d_scratch + off_recs)) != cudaSuccess)
        return cuda_fail(c, e, "anchor fits");
    if (clk_bytes && (st = prepare_clock(c, band, i0, n, b, (char *)((char *)c->d_scratch + off_eps)))) return st;
    if (split && (e = cudaStreamWaitEvent(c->stream, c->ev_join, 0)) != cudaSuccess) return cuda_fail(c, e, "join");
    prof_begin(c);
    if (split) {
        b.unocc_words = b.has_antenna ? d_uw : nullptr;
        e = launch_split_fanout(c->split_variant, b, c->d_tx, d_active, n_active, (char *)c->d_scratch + off_recs,
                                (float2 *)d_out, nullptr, nullptr, nullptr, c->stream);
    }
    else if (band->solver == LPK_SOLVER_FP64_TUNED)
        e = launch_band_fp64(b, c->d_tx, d_active, n_active, (float2 *)d_out, d_uw, c->stream);
    else
        e = launch_band_reference(b, c->d_tx, d_active, n_active, (float2 *)d_out, d_uw, c->stream);
    prof_end(c);
    c->launches += (n > 0) * (split ? 2 : 1);
    if (e != cudaSuccess) return cuda_fail(c, e, "fan-out kernel launch");
    if (d_unocc && n_active > 0) {
        c->launches += 1;
        e = launch_or_flags(d_uw, d_unocc, n_active, b.has_antenna ? 0 : (n > 0 ? 1 : 2), c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "occlusion flags");
    }
    return LPK_OK;
}

lpk_status lpk_split_accuracy(lpk_ctx *c, const lpk_band_desc *band, const int32_t *active, int32_t n_active,
                              int64_t i0, int64_t n, const double *d_delta, lpk_cf32 *d_out, double *max_delay_err_s,
                              double *max_phase_err_rad, int64_t *n_fast, int64_t *n_exact) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (!band || !use_split(band))
        return fail(c, LPK_EINVAL, "accuracy mode needs a split-solver band with a stationary or orbiting receiver");
    if (!max_delay_err_s || !max_phase_err_rad || !n_fast || !n_exact)
        return fail(c, LPK_EINVAL, "accuracy outputs are NULL");
    DevBand b;
    lpk_status st = build_dev_band(c, band, i0, n, b);
    if (st) return st;
    if ((st = check_active(c, active, n_active))) return st;
    if (b.clock_mode == LPK_CLOCK_HOST && n > 0 && !d_delta) return fail(c, LPK_EINVAL, "delta_t is NULL");
    b.delta = d_delta;
    cudaSetDevice(c->device);
    const size_t off_stats = align256(sizeof(int32_t) * 256);
    const size_t off_out = off_stats + 256;
    const size_t off_eps = off_out + (d_out ? 0 : align256(sizeof(float2) * (size_t)(n > 0 ? n : 0)));
    const size_t clk_bytes = clock_region_bytes(band, i0, n);
    const size_t off_recs = off_eps + clk_bytes;
    if ((st = ensure_scratch(c, off_recs + align256(split_recs_bytes(c->split_variant, i0, n, n_active)))))
        return st;
    char *base = (char *)c->d_scratch;
    int32_t *d_active = (int32_t *)base;
    unsigned long long *d_stats = (unsigned long long *)(base + off_stats);
    float2 *out = d_out ? (float2 *)d_out : (float2 *)(base + off_out);
    cudaError_t e = cudaMemcpyAsync(d_active, active, sizeof(int32_t) * (size_t)n_active, cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_stats, 0, 4 * sizeof(unsigned long long), c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "accuracy setup");
    if ((e = split_fork_anchor(c, b, d_active, n_active, base + off_recs)) != cudaSuccess)
        return cuda_fail(c, e, "anchor fits");
    if (clk_bytes && (st = prepare_clock(c, band, i0, n, b, (char *)(base + off_eps)))) return st;
    if ((e = cudaStreamWaitEvent(c->stream, c->ev_join, 0)) != cudaSuccess) return cuda_fail(c, e, "join");
    b.acc_stats = d_stats;
    e = launch_split_fanout(c->split_variant, b, c->d_tx, d_active, n_active, base + off_recs, out, nullptr, nullptr,
                            nullptr, c->stream);
    c->launches += (n > 0) * 2;
    if (e != cudaSuccess) return cuda_fail(c, e, "accuracy fan-out launch");
    unsigned long long h[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(h, d_stats, sizeof h, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "accuracy fan-out");
    double dd, dp;
    memcpy(&dd, &h[0], sizeof dd);
    memcpy(&dp, &h[1], sizeof dp);
    *max_delay_err_s = dd;
    *max_phase_err_rad = dp;
    *n_fast = (int64_t)h[2];
    *n_exact = (int64_t)h[3];
    return LPK_OK;
}

lpk_status lpk_sync(lpk_ctx *c) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "stream synchronize");
    return LPK_OK;
}

lpk_status lpk_band_chunk(lpk_ctx *c, const lpk_band_desc *band, const int32_t *active, int32_t n_active,
                          int64_t i0, int64_t n, const double *delta_t, const double *rx_pos3n, lpk_cf32 *out,
                          uint8_t *unoccluded) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    DevBand b;
    lpk_status st = build_dev_band(c, band, i0, n, b);
    if (st) return st;
    if ((st = check_active(c, active, n_active))) return st;
    if (b.clock_mode == LPK_CLOCK_HOST && n > 0 && !delta_t) return fail(c, LPK_EINVAL, "delta_t is NULL");
    if (b.rx_kind == LPK_RX_PER_SAMPLE && n > 0 && !rx_pos3n) return fail(c, LPK_EINVAL, "rx_pos3n is NULL");
    if (n > 0 && !out) return fail(c, LPK_EINVAL, "out is NULL");
    cudaSetDevice(c->device);
    size_t off_active = 0;
    size_t off_uw = align256(sizeof(int32_t) * 256);
    size_t off_delta = off_uw + align256(sizeof(uint32_t) * 256);
    size_t n_delta = b.clock_mode == LPK_CLOCK_HOST ? (size_t)n : 0;
    size_t off_rx = off_delta + align256(sizeof(double) * n_delta);
    size_t n_rx = b.rx_kind == LPK_RX_PER_SAMPLE ? 3 * (size_t)n : 0;
    size_t off_out = off_rx + align256(sizeof(double) * n_rx);
    size_t off_eps = off_out + align256(sizeof(float2) * (size_t)n);
    const size_t clk_bytes = clock_region_bytes(band, i0, n);
    const bool split = use_split(band);
    size_t off_recs = off_eps + clk_bytes;
    size_t total = off_recs + (split ? align256(split_recs_bytes(c->split_variant, i0, n, n_active)) : 0);
    if ((st = ensure_scratch(c, total))) return st;
    char *base = (char *)c->d_scratch;
    int32_t *d_active = (int32_t *)(base + off_active);
    uint32_t *d_uw = (uint32_t *)(base + off_uw);
    double *d_delta = (double *)(base + off_delta);
    double *d_rx = (double *)(base + off_rx);
    float2 *d_out = (float2 *)(base + off_out);
    cudaError_t e = cudaMemcpyAsync(d_active, active, sizeof(int32_t) * (size_t)n_active, cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_uw, 0, sizeof(uint32_t) * 256, c->stream);
    if (e == cudaSuccess && n_delta)
        e = cudaMemcpyAsync(d_delta, delta_t, sizeof(double) * n_delta, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && n_rx)
        e = cudaMemcpyAsync(d_rx, rx_pos3n, sizeof(double) * n_rx, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "chunk upload");
    b.delta = d_delta;
    b.rxpos = d_rx;
    if (split && (e = split_fork_anchor(c, b, d_active, n_active, base + off_recs)) != cudaSuccess)
        return cuda_fail(c, e, "anchor fits");
    if (clk_bytes && (st = prepare_clock(c, band, i0, n, b, (char *)(base + off_eps)))) return st;
    if (split && (e = cudaStreamWaitEvent(c->stream, c->ev_join, 0)) != cudaSuccess) return cuda_fail(c, e, "join");
    prof_begin(c);
    if (split) {
        b.unocc_words = b.has_antenna ? d_uw : nullptr;
        e = launch_split_fanout(c->split_variant, b, c->d_tx, d_active, n_active, base + off_recs, d_out, nullptr,
                                nullptr, nullptr, c->stream);
    }
    else if (band->solver == LPK_SOLVER_FP64_TUNED)
        e = launch_band_fp64(b, c->d_tx, d_active, n_active, d_out, d_uw, c->stream);
    else
        e = launch_band_reference(b, c->d_tx, d_active, n_active, d_out, d_uw, c->stream);
    prof_end(c);
    c->launches += (n > 0) * (split ? 2 : 1);
    if (e != cudaSuccess) return cuda_fail(c, e, "fan-out kernel launch");
    if (n > 0) e = cudaMemcpyAsync(out, d_out, sizeof(float2) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    uint32_t uw[256];
    if (e == cudaSuccess && unoccluded && n_active > 0)
        e = cudaMemcpyAsync(uw, d_uw, sizeof(uint32_t) * (size_t)n_active, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "fan-out kernel");
    if (unoccluded)
        for (int32_t k = 0; k < n_active; ++k)
            unoccluded[k] |= (uint8_t)(b.has_antenna ? (uw[k] != 0) : (n > 0));
    return LPK_OK;
}

lpk_status lpk_solve_emission_times(lpk_ctx *c, int32_t tx, const double *obs3n, const double *t_rel_utc,
                                    int64_t n, double epoch, int32_t iterations, double *t_emit,
                                    double *ranges) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (tx < 0 || tx >= c->n_tx) return fail(c, LPK_EINVAL, "transmitter index out of range");
    if (n < 0 || iterations < 0 || iterations > 64) return fail(c, LPK_EINVAL, "bad n or iterations");
    if (n == 0) return LPK_OK;
    if (!obs3n || !t_rel_utc || !t_emit || !ranges) return fail(c, LPK_EINVAL, "NULL array");
    cudaSetDevice(c->device);
    size_t bytes = sizeof(double) * (size_t)n;
    lpk_status st = ensure_scratch(c, 6 * bytes + 1024);
    if (st) return st;
    double *d_obs = (double *)c->d_scratch, *d_t = d_obs + 3 * n, *d_te = d_t + n, *d_r = d_te + n;
    cudaError_t e = cudaMemcpyAsync(d_obs, obs3n, 3 * bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_t, t_rel_utc, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = launch_solve(c->d_tx, tx, d_obs, d_t, n, epoch, iterations, 1.0 / kSpeedOfLight, d_te, d_r, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t_emit, d_te, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ranges, d_r, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "emission solve");
    return LPK_OK;
}

lpk_status lpk_tx_contribution(lpk_ctx *c, const lpk_band_desc *band, int32_t tx, int64_t i0, int64_t n,
                               const double *delta_t, const double *rx_pos3n, lpk_cf32 *out, double *phase_out,
                               double *t_emit_out, double *range_out) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (tx < 0 || tx >= c->n_tx) return fail(c, LPK_EINVAL, "transmitter index out of range");
    DevBand b;
    lpk_status st = build_dev_band(c, band, i0, n, b);
    if (st) return st;
    if (b.clock_mode == LPK_CLOCK_HOST && n > 0 && !delta_t) return fail(c, LPK_EINVAL, "delta_t is NULL");
    if (b.rx_kind == LPK_RX_PER_SAMPLE && n > 0 && !rx_pos3n) return fail(c, LPK_EINVAL, "rx_pos3n is NULL");
    if (n == 0) return LPK_OK;
    if (!out) return fail(c, LPK_EINVAL, "out is NULL");
    cudaSetDevice(c->device);
    size_t bytes = sizeof(double) * (size_t)n;
    const bool split = use_split(band);
    const size_t clk_bytes = clock_region_bytes(band, i0, n);
    size_t off_act = 8 * bytes;
    size_t off_eps = off_act + 256;
    size_t off_recs = off_eps + clk_bytes;
    const size_t recs_bytes = split ? align256(split_recs_bytes(c->split_variant, i0, n, 1)) : 0;
    lpk_status s2 = ensure_scratch(c, off_recs + recs_bytes + 256);
    if (s2) return s2;
    double *d_delta = (double *)c->d_scratch;
    double *d_rx = d_delta + n;
    double *d_phase = d_rx + 3 * n;
    double *d_te = d_phase + n;
    double *d_r = d_te + n;
    float2 *d_out = (float2 *)(d_r + n);
    char *base = (char *)c->d_scratch;
    cudaError_t e = cudaSuccess;
    if (b.clock_mode == LPK_CLOCK_HOST) e = cudaMemcpyAsync(d_delta, delta_t, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && b.rx_kind == LPK_RX_PER_SAMPLE)
        e = cudaMemcpyAsync(d_rx, rx_pos3n, 3 * bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + off_act, &tx, sizeof(int32_t), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "transmitter contribution upload");
    b.delta = d_delta;
    b.rxpos = d_rx;
    if (clk_bytes && (s2 = prepare_clock(c, band, i0, n, b, (char *)(base + off_eps)))) return s2;
    if (split) {
        b.has_noise = 0;  // the contribution alone, as transmitter_contribution_at_receiver returns it
        b.n_post = 0;
        e = launch_band_split(c->split_variant, b, c->d_tx, (const int32_t *)(base + off_act), 1, base + off_recs,
                              d_out, d_phase, d_te,
                              d_r, c->stream);
    } else {
        e = launch_tx_contribution(b, c->d_tx, tx, d_out, d_phase, d_te, d_r, c->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, sizeof(float2) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && phase_out)
        e = cudaMemcpyAsync(phase_out, d_phase, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && t_emit_out) e = cudaMemcpyAsync(t_emit_out, d_te, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && range_out) e = cudaMemcpyAsync(range_out, d_r, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "transmitter contribution");
    if (split && range_out)  // the split kernel reports delay; range = c · delay
        for (int64_t i = 0; i < n; ++i) range_out[i] *= kSpeedOfLight;
    return LPK_OK;
}

lpk_status lpk_sample_times(lpk_ctx *c, double fs_hz, int64_t i0, int64_t n, double *t_out) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (!(fs_hz > 0.0) || !std::isfinite(fs_hz)) return fail(c, LPK_EINVAL, "fs_hz must be positive and finite");
    if (n < 0 || i0 < 0 || i0 > ((int64_t)1 << 53) - n) return fail(c, LPK_EINVAL, "bad sample range");
    if (n == 0) return LPK_OK;
    if (!t_out) return fail(c, LPK_EINVAL, "t_out is NULL");
    cudaSetDevice(c->device);
    lpk_status st = ensure_scratch(c, sizeof(double) * (size_t)n);
    if (st) return st;
    cudaError_t e = launch_sample_times(fs_hz, i0, n, (double *)c->d_scratch, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(t_out, c->d_scratch, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? LPK_OK : cuda_fail(c, e, "sample times");
}

lpk_status lpk_clock_device_delta(lpk_ctx *c, const lpk_band_desc *band, int64_t i0, int64_t n, double *out) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    DevBand b;
    lpk_status st = build_dev_band(c, band, i0, n, b);
    if (st) return st;
    if (b.clock_mode == LPK_CLOCK_HOST) return fail(c, LPK_EINVAL, "host clock mode has no device Δt");
    if (n == 0) return LPK_OK;
    if (!out) return fail(c, LPK_EINVAL, "delta_out is NULL");
    cudaSetDevice(c->device);
    const size_t clk_bytes = clock_region_bytes(band, i0, n);
    size_t off_eps = align256(sizeof(double) * (size_t)n);
    if ((st = ensure_scratch(c, off_eps + clk_bytes))) return st;
    double *d_out = (double *)c->d_scratch;
    if (clk_bytes && (st = prepare_clock(c, band, i0, n, b, (char *)((char *)c->d_scratch + off_eps)))) return st;
    cudaError_t e = launch_band_delta(b, d_out, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "device clock");
    return LPK_OK;
}

lpk_status lpk_rx_chain_apply(lpk_ctx *c, const lpk_band_desc *band, lpk_cf32 *iq, int64_t n) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    lpk_band_desc d = band ? *band : lpk_band_desc{};
    d.noise_power_w = 0.0;
    d.clock_mode = LPK_CLOCK_DETERMINISTIC;
    DevBand b;
    lpk_status st = build_dev_band(c, band ? &d : nullptr, 0, n, b);
    if (st) return st;
    if (n == 0) return LPK_OK;
    if (!iq) return fail(c, LPK_EINVAL, "iq is NULL");
    cudaSetDevice(c->device);
    if ((st = ensure_scratch(c, sizeof(float2) * (size_t)n))) return st;
    float2 *d_iq = (float2 *)c->d_scratch;
    cudaError_t e = cudaMemcpyAsync(d_iq, iq, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_rx_chain(b, d_iq, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(iq, d_iq, sizeof(float2) * (size_t)n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "rx chain");
    return LPK_OK;
}

}  // extern "C"
