/*
 * lipika_cuda.h — C ABI of the B200 (sm_100a) IQ-generation backend.
 *
 * The boundary replaces the per-chunk transmitter fan-out of the reference
 * and everything after the transmitter sum, src/pipeline.rs:943-983:
 *   gated_contribution -> accumulate_reporting_occlusion (channel/mod.rs:164-271)
 *   fixed-order reduction                                 (pipeline.rs:966-977)
 *   add_awgn_at_power                                      (channel/mod.rs:323-334)
 *   RxChain::apply_post_sum                                (rx/mod.rs:142-146)
 * The chunk loop, the clock stream and the sinks stay in the host.
 *
 * Conventions (all entry points):
 *   - plain C types and pointers only; no CUDA or torch types cross the ABI;
 *   - every call returns an lpk_status (0 = OK, negative = error) and never
 *     aborts or exits; lpk_last_error() holds a message for the last failure;
 *   - host pointers are borrowed for the duration of the call only; the
 *     library copies what it keeps into memory owned by the lpk_ctx;
 *   - one lpk_ctx per host thread: calls on different contexts are
 *     thread-safe, calls on one context must be serialised (the reference
 *     calls generate_band concurrently from rayon workers,
 *     src/pipeline.rs:513-535, each with its own state).
 */
#ifndef LIPIKA_CUDA_H
#define LIPIKA_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "lipika_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t lpk_status;
#define LPK_OK 0
#define LPK_EINVAL (-1)     /* bad descriptor, NaN or out-of-range configuration */
#define LPK_ENOMEM (-2)     /* host or device allocation failed */
#define LPK_ECUDA (-3)      /* a CUDA call failed; lpk_last_error() has its string */
#define LPK_ETIMEDOUT (-4)  /* a bounded device wait gave up */
#define LPK_ENOCONV (-5)    /* an emission solve did not converge */
#define LPK_ENOTSUP (-6)    /* feature outside this backend (TLE, RINEX, LNAV) */

typedef struct lpk_ctx lpk_ctx;
typedef struct lpk_cf32 { float re, im; } lpk_cf32;

/* ------------------------------------------------------------------ */
/* Context                                                             */
/* ------------------------------------------------------------------ */
/* Create a context bound to CUDA device `device` (own stream + buffers).
 * Replaces: Backend::Cpu selection, src/backend/mod.rs:16-18. */
lpk_status lpk_ctx_create(lpk_ctx **out, int32_t device);
/* Destroy every scene, batch and network made on a context before the
 * context: their handles refer to it. */
void lpk_ctx_destroy(lpk_ctx *ctx);
/* Message of the last failed call on this context ("" if none). */
const char *lpk_last_error(const lpk_ctx *ctx);
/* Message of the last failure that happened before a context existed. */
const char *lpk_global_last_error(void);
/* Library version string. */
const char *lpk_version(void);
/* The context's CUDA stream as an opaque handle (a cudaStream_t), so a
 * host can order its own work or timing events against the library's. */
void *lpk_ctx_stream(lpk_ctx *ctx);

/* Measurement hooks (no reference counterpart; the reference times coarse
 * sections with profile::time, src/profile.rs:27-36). While enabled, every
 * fan-out launch is bracketed by CUDA events on the context's stream.
 * lpk_profile_read waits for the stream, then reports the summed fan-out
 * kernel time, the number of fan-out launches and the number of all kernel
 * launches since the last reset. */
lpk_status lpk_profile_enable(lpk_ctx *ctx, int32_t on);
lpk_status lpk_profile_reset(lpk_ctx *ctx);
lpk_status lpk_profile_read(lpk_ctx *ctx, double *fanout_ms, int64_t *fanout_launches,
                            int64_t *all_launches);
/* Horizon gate counters of this context (src/channel/horizon.rs): with an
 * antenna cutoff, each block of band samples (256 in the FP64 kernel, one
 * tile in the split and batched kernels) tests every transmitter with the
 * reference's certainly_below_cutoff bound and skips those certainly below
 * the cutoff for all its samples (their contribution is zero either way).
 * `tested` (block, transmitter) pairs, `skipped` of them; reset != 0
 * clears both afterwards. */
lpk_status lpk_gate_stats(lpk_ctx *ctx, int64_t *tested, int64_t *skipped, int32_t reset);
/* Measured FP64 FMA throughput of the device (TFLOP/s, 2 flops per FMA)
 * from a register-resident DFMA chain kernel timed with CUDA events. */
lpk_status lpk_probe_fp64_peak(lpk_ctx *ctx, double *tflops);

/* ------------------------------------------------------------------ */
/* Kernel-level boundary: transmitters as already-built tables          */
/* ------------------------------------------------------------------ */
enum { LPK_TX_TRAJ_STATIONARY = 0, LPK_TX_TRAJ_PRECOMPUTED = 1 };

/* One transmitter as the reference's host holds it after prepare():
 * AnyTrajectory::{Stationary, Precomputed} (geometry/mod.rs:25-31,
 * precomputed.rs:157-172) + a SignalModel (src/signal/) + EIRP.
 * Tables are host pointers, copied by lpk_scene_upload. */
typedef struct lpk_tx_desc {
    int32_t traj_kind;          /* LPK_TX_TRAJ_* */
    int32_t sig_kind;           /* LPK_SIG_* (lipika_scene.h) */
    double stationary_ecef[3];
    double grid_t0_unix;        /* PrecomputedTrajectory::t0_unix */
    double grid_dt_s;           /* ::dt_s */
    int64_t grid_n;             /* ::n */
    const double *grid_xyz;     /* (3, grid_n) axis-major, as ndarray holds it */
    double carrier_hz;          /* SignalModel::carrier_hz */
    double tx_power_w;          /* 10^(dBW/10), pipeline.rs:338 */
    /* framed kinds (bpsk, ook, qam16) and ca_code */
    double epoch_rel_s;         /* symbol/chip-0 tag, scene-epoch relative */
    double rate_hz;             /* bit or symbol rate (framed kinds) */
    int32_t has_repeat;         /* repeat_from is Some */
    int32_t nav_kind;           /* ca_code: LPK_NAV_* */
    int64_t repeat_from;
    int64_t n_sym;              /* frame length */
    const int8_t *pm_bits;      /* bpsk: n_sym values ±1 */
    const uint8_t *ook_bits;    /* ook: n_sym values 0/1 */
    const lpk_cf32 *symbols;    /* qam16: n_sym constellation points */
    const int8_t *chips;        /* ca_code: 1023 values ±1 */
    uint64_t nav_seed;          /* dummy nav: folded seed (ca_code.rs:148-149) */
    const int8_t *nav_bits;     /* full nav: nav_n values ±1 */
    int64_t nav_n;
    /* cw */
    double cw_offset_hz;
    double cw_phase0;           /* anchored phase (cw.rs:22-34) */
    int32_t cw_anchored;
    /* burst gate (gate.rs:27-34) */
    int32_t has_gate;
    double gate_period_s;
    double gate_phase_s;
    int32_t gate_n;
    int32_t reserved;
    const double *gate_on;      /* gate_n (start, end) pairs */
} lpk_tx_desc;

/* Upload the scene's transmitters (replaces the host-side Vec<Transmitter>
 * the fan-out reads, src/pipeline.rs:297-342). Replaces any earlier upload. */
lpk_status lpk_scene_upload(lpk_ctx *ctx, const lpk_tx_desc *tx, int32_t n_tx);

/* Trajectory tables of circular Keplerian orbits built on the GPU: replaces
 * PrecomputedTrajectory::sample over CircularKeplerian::position_ecef
 * (src/geometry/precomputed.rs:47-70, src/geometry/kepler.rs:32-85) for a
 * set of orbits sharing one grid. For each orbit, the ECEF positions at
 * t0_unix + i dt_s (i < n_points) are written to grid_xyz (host memory) as
 * n_orbits consecutive (3, n_points) axis-major blocks, the layout of
 * lpk_tx_desc.grid_xyz. FP64 with the host's operation order; the per-orbit
 * constants come from the host's libm and the per-point sines and cosines
 * from the GPU's, so an entry may differ from a host-built table in its
 * last bits (~1e-9 m). */
typedef struct lpk_kepler_orbit {
    double semi_major_axis_m, inclination_deg, raan_deg, true_anomaly_deg_at_epoch, epoch_unix;
} lpk_kepler_orbit;
lpk_status lpk_kepler_tables(lpk_ctx *ctx, const lpk_kepler_orbit *orbits, int32_t n_orbits, double t0_unix,
                             double dt_s, int64_t n_points, double *grid_xyz);

enum { LPK_CLOCK_HOST = 0, LPK_CLOCK_DETERMINISTIC = 1, LPK_CLOCK_DEVICE_WALK = 2 };
/* LPK_RX_KEPLER: a receiver on a circular Keplerian orbit (lpk_band_desc
 * rx_orbit), positioned on the device at each sample's rounded absolute UTC
 * time exactly as receiver.trajectory.position_ecef_batch(epoch + t_utc)
 * does (src/pipeline.rs:929-931, src/geometry/kepler.rs:32-85). */
enum { LPK_RX_STATIONARY = 0, LPK_RX_PER_SAMPLE = 1, LPK_RX_KEPLER = 2 };
enum { LPK_POST_GAIN = 0, LPK_POST_NONLINEARITY = 1, LPK_POST_ADC = 2 };
/* Fan-out solvers: REFERENCE, the reference's per-sample f64 arithmetic in
 * its order (bit-exact emission times, indices and ADC codes); SPLIT, the
 * split-precision fan-out (FP64 anchors per tile, FP32 mix; delay within
 * 1 ps, carrier phase within 1e-6 rad, IQ within 1e-5 of REFERENCE);
 * FP64_TUNED, the same two iterations all in FP64 with the shortcuts a tuned
 * FP64 kernel takes (table lerp scaled by 1/dt, carrier and CW phases
 * reduced modulo 2π before one FP64 sincos, f32 amplitude division; within
 * the IQ tolerance of REFERENCE; per-band entry points only, the batch runs
 * REFERENCE for it). */
enum { LPK_SOLVER_REFERENCE = 0, LPK_SOLVER_SPLIT = 1, LPK_SOLVER_FP64_TUNED = 2 };

typedef struct lpk_post_op {
    int32_t kind;               /* LPK_POST_* */
    uint32_t bits;              /* adc */
    double param;               /* gain_db | iip3_w | full_scale_v */
} lpk_post_op;

/* One (receiver, band) work unit's per-chunk parameters
 * (generate_band's locals, src/pipeline.rs:853-905). */
typedef struct lpk_band_desc {
    double epoch_unix;          /* scene epoch */
    double fs_hz;               /* band sample rate */
    double lo_hz;               /* band LO */
    double noise_power_w;       /* AWGN power; <= 0 disables noise */
    uint64_t noise_seed;        /* noise_seed(base, work_idx), pipeline.rs:828 */
    int32_t rx_kind;            /* LPK_RX_* */
    int32_t clock_mode;         /* LPK_CLOCK_* */
    double rx_ecef[3];          /* stationary receiver */
    /* clock (NodeClockSpec) for DETERMINISTIC / DEVICE_WALK modes */
    double clock_offset_s;
    double clock_y0;
    double clock_allan_1s;
    double clock_master_rate_hz;
    uint64_t clock_seed;        /* clock_seed(base, r_idx), pipeline.rs:825 */
    /* antenna (Antenna, rx/mod.rs:41-58) */
    int32_t has_antenna;
    int32_t has_cutoff;
    double ant_peak_dbi, ant_horizon_dbi, ant_fb_db, ant_cutoff_deg;
    /* post-sum chain (RxChain::post_sum, rx/mod.rs:117-146) */
    int32_t n_post;
    int32_t solver;             /* LPK_SOLVER_* */
    lpk_post_op post[3];
    /* Flicker-FM part of the clock (Flicker, src/clock/mod.rs:55-149) for
     * the DETERMINISTIC and DEVICE_WALK modes: the coarse flicker track D[m]
     * at m / 128 s of local time, m = 0..flicker_n-1, in HOST memory
     * (lpk_clock_flicker_table; the host stream interpolates it linearly,
     * Flicker::delta_at, :142-148, and so do the kernels). NULL: no
     * flicker. Ignored under LPK_CLOCK_HOST, whose Δt already holds it.
     * lpk_scene_band_desc fills it for a clock with a flicker floor; the
     * scene owns that table. */
    const double *flicker_delta_s;
    int64_t flicker_n;
    lpk_kepler_orbit rx_orbit;  /* LPK_RX_KEPLER: the receiver's orbit */
} lpk_band_desc;

/* One chunk of one band through the fan-out, Σ, AWGN and rx chain.
 * Replaces src/pipeline.rs:943-983 for the chunk [i0, i0 + n).
 *   active_tx  : indices into the uploaded transmitters, in band order
 *                (the band-overlap gate's `active`, pipeline.rs:882-891)
 *   delta_t    : n clock offsets Δt (host), required for LPK_CLOCK_HOST
 *   rx_pos3n   : (3, n) receiver ECEF per sample (host), LPK_RX_PER_SAMPLE
 *   out        : n complex64 samples (host)
 *   unoccluded : n_active flags OR-ed with "non-zero antenna gain for at
 *                least one sample" (accumulate_reporting_occlusion's
 *                return value, channel/mod.rs:204-207); may be NULL. */
lpk_status lpk_band_chunk(lpk_ctx *ctx, const lpk_band_desc *band, const int32_t *active_tx,
                          int32_t n_active, int64_t i0, int64_t n, const double *delta_t,
                          const double *rx_pos3n, lpk_cf32 *out, uint8_t *unoccluded);

/* Same as lpk_band_chunk, but every array is DEVICE memory and the work is
 * only enqueued on the context's stream (call lpk_sync to wait). Used by
 * hosts that keep inputs and outputs resident in HBM. */
lpk_status lpk_band_chunk_device(lpk_ctx *ctx, const lpk_band_desc *band, const int32_t *active_tx,
                                 int32_t n_active, int64_t i0, int64_t n, const double *d_delta_t,
                                 const double *d_rx_pos3n, lpk_cf32 *d_out, uint8_t *d_unoccluded);
lpk_status lpk_sync(lpk_ctx *ctx);

/* Accuracy of the split-precision fan-out (no reference counterpart; the
 * reference has one all-FP64 path). Renders band samples [i0, i0 + n) of a
 * band with solver LPK_SOLVER_SPLIT and a stationary or orbiting receiver exactly as
 * lpk_band_chunk_device does (into d_out, DEVICE memory, when not NULL),
 * and for every (sample, transmitter) the split path evaluates on its fast
 * path also runs the reference-exact FP64 solve and phase (the arithmetic
 * of the all-FP64 kernel, src/channel/mod.rs:70-99, :251-267): returns the
 * largest |delay difference| (s) and |carrier-phase difference| (rad,
 * wrapped to [-pi, pi]) over them, the number of fast-path (sample,
 * transmitter) pairs compared and the number taken on the exact path
 * (which equal the FP64 kernel's by construction). Synchronous. */
lpk_status lpk_split_accuracy(lpk_ctx *ctx, const lpk_band_desc *band, const int32_t *active_tx, int32_t n_active,
                              int64_t i0, int64_t n, const double *d_delta_t, lpk_cf32 *d_out,
                              double *max_delay_err_s, double *max_phase_err_rad, int64_t *n_fast, int64_t *n_exact);

/* lpk_band_chunk_device for callers that cannot allocate device memory when
 * they render (a real-time thread that must not stall on the CUDA allocator,
 * a host that reserved the device for its own pool). No counterpart in the
 * reference. It calls no cudaMalloc/cudaFree: its working memory is one
 * file-scope static device array of 22.6 MiB that every GPU loading this
 * library holds until exit. It runs the kernels lpk_band_chunk_device runs
 * for the band's solver (the split path for LPK_SOLVER_SPLIT with a
 * stationary or orbiting receiver, the FP64 kernel otherwise) on the same
 * inputs, so
 * its outputs equal lpk_band_chunk_device's bit for bit. Limits: at most
 * 256 active transmitters; with LPK_CLOCK_DEVICE_WALK a chunk may span at
 * most 2^20 master-clock samples and lie within the first 2^29; a split
 * chunk may need at most 32,768 (tile, transmitter) anchor records and at
 * most 8,192 flicker-track points (larger requests return LPK_EINVAL). Every call rebuilds the clock walk's block
 * totals and carries from master sample 0, so its walk work grows with the
 * chunk's master-sample offset. The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) — make that first call before any
 * stream capture. All calls share the array: calls that overlap on the GPU
 * race; each call re-clears what it needs zeroed. */
lpk_status lpk_band_chunk_device_static(lpk_ctx *ctx, const lpk_band_desc *band, const int32_t *active_tx,
                                        int32_t n_active, int64_t i0, int64_t n, const double *d_delta_t,
                                        const double *d_rx_pos3n, lpk_cf32 *d_out, uint8_t *d_unoccluded);

/* Per-transmitter emission solve (channel/mod.rs:106-121,
 * solve_emission_times): `iterations` fixed-point steps from t - 70 ms.
 * All arrays host memory, obs3n is (3, n) axis-major. */
lpk_status lpk_solve_emission_times(lpk_ctx *ctx, int32_t tx, const double *obs3n,
                                    const double *t_rel_utc, int64_t n, double epoch,
                                    int32_t iterations, double *t_emit, double *ranges);

/* One transmitter's contribution alone (channel/mod.rs:278-298,
 * transmitter_contribution_at_receiver) for the band's chunk; optional
 * per-sample carrier phase reduced to [-pi, pi) (phase_out, may be NULL). */
lpk_status lpk_tx_contribution(lpk_ctx *ctx, const lpk_band_desc *band, int32_t tx, int64_t i0,
                               int64_t n, const double *delta_t, const double *rx_pos3n,
                               lpk_cf32 *out, double *phase_out, double *t_emit_out,
                               double *range_out);

/* The clock offsets Δt the fan-out uses for band samples [i0, i0 + n) under
 * the band's clock mode (DETERMINISTIC or DEVICE_WALK), copied to host
 * memory: ClockStream::delta_t_at (src/clock/mod.rs:329-346) evaluated on
 * the device. */
lpk_status lpk_clock_device_delta(lpk_ctx *ctx, const lpk_band_desc *band, int64_t i0, int64_t n,
                                  double *delta_out);

/* The local sample times t = i / fs_hz (src/pipeline.rs:918: `i as f64 / fs`)
 * for i in [i0, i0 + n) exactly as the split fan-out forms them on the
 * device (a reciprocal, a product and one fma correction instead of a
 * division), copied to host memory; they must equal the IEEE quotient. */
lpk_status lpk_sample_times(lpk_ctx *ctx, double fs_hz, int64_t i0, int64_t n, double *t_out);

/* AWGN-free rx chain alone on n samples in place (RxChain::apply_post_sum,
 * src/rx/mod.rs:142-146): the band's post ops on caller-supplied f32 IQ,
 * so ADC codes can be compared on identical inputs. Host memory. */
lpk_status lpk_rx_chain_apply(lpk_ctx *ctx, const lpk_band_desc *band, lpk_cf32 *iq, int64_t n);

/* ------------------------------------------------------------------ */
/* Launch shapes of the split-precision fan-out                        */
/* ------------------------------------------------------------------ */
/* The split kernel is compiled in several launch shapes (band samples per
 * tile, threads per block, minimum resident blocks per SM). No reference
 * counterpart: the reference has one CPU loop. */
int32_t lpk_split_variant_count(void);
lpk_status lpk_split_variant_info(int32_t variant, int32_t *tile, int32_t *threads, int32_t *min_blocks);
/* Shape used by this context's single-band entry points (default 0). */
lpk_status lpk_ctx_set_split_variant(lpk_ctx *ctx, int32_t variant);
int32_t lpk_ctx_split_variant(const lpk_ctx *ctx);

/* ------------------------------------------------------------------ */
/* Batched fan-out: every (receiver, band) work unit in one launch     */
/* ------------------------------------------------------------------ */
/* Replaces the per-work-unit loop of run_scene_to_dir / run_scene_in_memory
 * (src/pipeline.rs:460-536: one generate_band per (rx, band), run by rayon
 * workers) for a whole scene at once. Time advances in rounds of round_s
 * seconds: in round k unit u renders band samples [k L_u, (k+1) L_u) with
 * L_u = llround(round_s * fs_u), clipped to its length, so units of uneven
 * rate and length progress together. One round is one CUDA graph (a copy of
 * the round's descriptor, the clock walks of every receiver, the anchor
 * fits of every (unit, tile, transmitter), and one persistent fan-out kernel
 * that pulls tiles of every unit from a shared counter); the graph is built
 * once and replayed. Outputs equal the single-band entry points' for the
 * same solver and split launch shape (chunk invariance).
 * Units need a stationary or orbiting receiver (rx_kind LPK_RX_STATIONARY
 * or LPK_RX_KEPLER) and a clock mode of LPK_CLOCK_DETERMINISTIC or
 * LPK_CLOCK_DEVICE_WALK (with or without a flicker track); units whose
 * clock seed, master rate and Allan deviation agree share one walk (the
 * bands of one receiver). Units with solver LPK_SOLVER_REFERENCE take the
 * reference-exact path for every sample. */
typedef struct lpk_batch lpk_batch;
typedef struct lpk_work_unit {
    lpk_band_desc band;
    const int32_t *active;   /* in-band transmitters, summed in this order (host memory) */
    int32_t n_active;
    int32_t reserved;
    int64_t n_samples;       /* band length */
} lpk_work_unit;

lpk_status lpk_batch_create(lpk_ctx *ctx, const lpk_work_unit *units, int32_t n_units, double round_s,
                            lpk_batch **out);
void lpk_batch_destroy(lpk_batch *b);
int64_t lpk_batch_n_rounds(const lpk_batch *b);
/* Band samples [*i0, *i0 + *n) of unit `unit` in round `round`. */
lpk_status lpk_batch_round_extent(const lpk_batch *b, int64_t round, int32_t unit, int64_t *i0, int64_t *n);
/* Enqueue round `round` on the context's stream (asynchronous). Rounds may
 * run in any order; the walk carries they need are completed on the way. */
lpk_status lpk_batch_run(lpk_batch *b, int64_t round);
/* Device pointer of unit `unit`'s output of the last round run (valid until
 * the next lpk_batch_run). */
lpk_status lpk_batch_output(lpk_batch *b, int32_t unit, const lpk_cf32 **d_out);
/* Wait for the last round and copy unit `unit`'s output to host memory. */
lpk_status lpk_batch_copy_out(lpk_batch *b, int32_t unit, lpk_cf32 *host, int64_t cap);
/* Forget the clock-walk carries computed so far, so the next rounds redo
 * all the walk work a fresh batch would (outputs are unchanged). */
lpk_status lpk_batch_reset(lpk_batch *b);
/* Sink of lpk_batch_render / lpk_generate_scene: one unit's chunk, in
 * order; return 0 to continue, 1 to stop that unit, negative to abort. */
typedef int32_t (*lpk_unit_sink_fn)(void *user, int32_t unit, const lpk_cf32 *chunk, int64_t n);
/* Every round in order with the outputs double-buffered: while round k
 * renders, round k-1's outputs are copied to pinned host staging on a
 * second stream and handed to sink(user, unit, chunk, n) (the chunk points
 * into the staging; valid during the call). */
lpk_status lpk_batch_render(lpk_batch *b, lpk_unit_sink_fn sink, void *user);
/* Launch configuration: split shape and persistent blocks per SM (0 = the
 * most that fit). */
lpk_status lpk_batch_set_config(lpk_batch *b, int32_t variant, int32_t blocks_per_sm);
lpk_status lpk_batch_get_config(const lpk_batch *b, int32_t *variant, int32_t *blocks_per_sm,
                                int32_t *max_blocks_per_sm);
/* Autotuner: run round `round` under every (variant, blocks per SM) pair
 * the device can hold (blocks per SM: the maximum, and half of it),
 * `reps` timed replays each after one warm-up, keep the fastest. ms_table
 * (may be NULL) receives lpk_split_variant_count() x 2 mean milliseconds
 * per round (negative where a pair was skipped). */
lpk_status lpk_batch_autotune(lpk_batch *b, int64_t round, int32_t reps, double *ms_table);

/* ------------------------------------------------------------------ */
/* Converged emission solve and its learned warm start                 */
/* ------------------------------------------------------------------ */
/* The reference stops after two fixed-point iterations from t - 70 ms
 * (src/channel/mod.rs:49-101, NEWTON_ITERATIONS = 2), which is what the
 * fan-out reproduces. lpk_solve_converged instead iterates to a tolerance
 * (the delay truth the reference's own tests compare against,
 * src/channel/mod.rs:355-383, runs four iterations), on the same
 * trajectory model (lerp table, linearised Sagnac), from one of three
 * starts: the reference's t - 70 ms (LAG), the range at the reception time
 * from the trajectory table R(t)/c (GEOMETRIC), or the scene's surrogate
 * (LEARNED, see lpk_mlp below). A start that does not converge within
 * max_iter falls back to LAG; iters[i] counts every map evaluation (-1 if
 * even the fallback did not converge) and start_err[i] (may be NULL) is
 * |start - converged delay| in seconds. No reference counterpart. */
enum { LPK_START_LAG = 0, LPK_START_GEOMETRIC = 1, LPK_START_LEARNED = 2 };
enum { LPK_ITER_FIXED_POINT = 0, LPK_ITER_NEWTON = 1 };
#define LPK_MLP_N_FEATURES 16
#define LPK_MLP_N_PARAMS 9473  /* W1 64x16, b1 64, W2 64x64, b2 64, W3 64x64, b3 64, w4 64, b4 (FP32, row-major) */
#define LPK_MLP_N_NORM 34      /* feature means (16), feature stds (16), target mean, target std (µs) */
typedef struct lpk_mlp lpk_mlp;

lpk_status lpk_solve_converged(lpk_ctx *ctx, int32_t tx, const double *rx_ecef, double epoch,
                               const double *t_rel_utc, int64_t n, double tol_s, int32_t max_iter,
                               int32_t scheme, int32_t start, const lpk_mlp *mlp, double *t_emit,
                               int32_t *iters, float *start_err);
/* The same over many (transmitter, receiver) pairs at once: sample i solves
 * transmitter tx[i] for receiver rx_ecef[3 rx[i] .. 3 rx[i] + 2] (n_rx
 * receivers). device_ms (may be NULL) receives the device time of the
 * call's kernels (features, network and solve; CUDA events on the
 * context's stream, host copies excluded). Host memory. */
lpk_status lpk_solve_converged_scene(lpk_ctx *ctx, const int32_t *tx, const int32_t *rx, const double *rx_ecef,
                                     int32_t n_rx, double epoch, const double *t_rel_utc, int64_t n, double tol_s,
                                     int32_t max_iter, int32_t scheme, int32_t start, const lpk_mlp *mlp,
                                     double *t_emit, int32_t *iters, float *start_err, double *device_ms);
/* The scene's surrogate of the emission delay: a function of a
 * transmitter's circular-orbit elements (lpk_kepler_orbit), a receiver's
 * ECEF position and the reception time t (scene-epoch relative) alone. An
 * analytic layer turns them into 16 features (the elements a, inclination,
 * RAAN and true anomaly at epoch; the receiver's x, y, z; t; and, from the
 * orbit at t: the line-of-sight unit vector, R/c, range rate / c, v_x / c,
 * v_y / c and the Sagnac rate of the line of sight); a tanh MLP
 * 16 -> 64 -> 64 -> 64 -> 1 predicts from them, normalised, the light-time
 * correction tau - R/c (µs); the learned start is R/c plus that correction.
 * One network covers every (transmitter, receiver) pair of a scene.
 * Glorot-uniform initial weights from `seed`. Inference runs on tcgen05
 * tensor cores (BF16 operands, FP32 accumulator in TMEM); training's
 * products are BF16 mma.sync tiles with FP32 accumulation; Adam updates
 * FP32 master weights. */
lpk_status lpk_mlp_create(lpk_ctx *ctx, uint64_t seed, lpk_mlp **out);
void lpk_mlp_destroy(lpk_mlp *mlp);
lpk_status lpk_mlp_get_params(const lpk_mlp *mlp, float *params, float *norm);
lpk_status lpk_mlp_set_params(lpk_mlp *mlp, const float *params, const float *norm);
/* The network's transmitters: tx[k] (uploaded scene indices, moving) with
 * circular orbit orbits[k]. lpk_mlp_fit sets them; a network restored with
 * lpk_mlp_set_params needs them before it can serve a learned start. */
lpk_status lpk_mlp_set_orbits(lpk_mlp *mlp, const int32_t *tx, const lpk_kepler_orbit *orbits, int32_t n_tx);
/* y = MLP(x) on n rows of normalised features (host memory). */
lpk_status lpk_mlp_forward(lpk_mlp *mlp, const float *x, int64_t n, float *y);
/* Mean squared error over n rows and its gradient (LPK_MLP_N_PARAMS floats,
 * the parameter layout above); host memory. */
lpk_status lpk_mlp_loss_grad(lpk_mlp *mlp, const float *x, const float *t, int64_t n, double *loss,
                             float *grad);
/* Train on n_train (transmitter, receiver, reception time) triples: orbit k
 * and receiver j drawn uniformly (tx[k], orbits[k]; rx_ecef holds n_rx
 * positions), t uniform in [t0, t1). The converged Newton solver (started
 * at the orbit's R/c) produces the targets on the GPU, the normalisation
 * comes from the first 2^21 rows of the training set, then `steps` Adam
 * steps on batches of `batch` rows with a cosine-decayed learning rate.
 * loss_curve (may be NULL) receives each step's batch MSE in normalised
 * units. */
lpk_status lpk_mlp_fit(lpk_mlp *mlp, const int32_t *tx, const lpk_kepler_orbit *orbits, int32_t n_tx,
                       const double *rx_ecef, int32_t n_rx, double epoch, double t0, double t1, int64_t n_train,
                       int32_t steps, int32_t batch, float lr, uint64_t seed, float *loss_curve);
/* The network's 16 raw input features of transmitter tx (one of its
 * orbits) seen from rx_ecef at the reception times (n x 16, host memory). */
lpk_status lpk_mlp_features(const lpk_mlp *mlp, int32_t tx, const double *rx_ecef, double epoch,
                            const double *t_rel_utc, int64_t n, float *features);
/* Self-check of the inference kernel's bounded tensor-core completion wait
 * (no reference counterpart): runs the kernel on n rows with its MMAs
 * withheld, so every completion wait gives up after `spin` polls with
 * nothing in flight. Returns LPK_ETIMEDOUT when the give-up path reported
 * it (the expected outcome; the context stays usable), LPK_EINVAL if a wait
 * did not give up. */
lpk_status lpk_mlp_wait_selftest(lpk_mlp *mlp, int64_t n, int32_t spin);

/* ------------------------------------------------------------------ */
/* Host-level mirror of src/pipeline.rs (scene -> per-band streams)     */
/* ------------------------------------------------------------------ */
typedef struct lpk_scene lpk_scene;

/* prepare() (src/pipeline.rs:801-819): build every transmitter's
 * trajectory table and signal tables from the scene description, check
 * them, and upload them to ctx. The scene keeps a borrowed ctx pointer.
 * With ctx == NULL the tables are built and checked but not uploaded
 * (lpk_scene_tx_desc still works; nothing that launches work does). */
lpk_status lpk_scene_prepare(lpk_ctx *ctx, const lpk_scene_cfg *cfg, lpk_scene **out);
void lpk_scene_free(lpk_scene *s);
int32_t lpk_scene_n_work(const lpk_scene *s);
lpk_status lpk_scene_work(const lpk_scene *s, int32_t work_idx, int32_t *r_idx, int32_t *b_idx);
int64_t lpk_scene_band_samples(const lpk_scene *s, int32_t r_idx, int32_t b_idx);
/* Active (in-band) transmitter indices of a band; returns the count. */
int32_t lpk_scene_band_active(const lpk_scene *s, int32_t r_idx, int32_t b_idx, int32_t *active,
                              int32_t cap);
/* Copy transmitter tx's uploaded descriptor (tables stay owned by s). */
lpk_status lpk_scene_tx_desc(const lpk_scene *s, int32_t tx, lpk_tx_desc *out);
/* Fill the band descriptor generate_band would use for (r_idx, b_idx). */
lpk_status lpk_scene_band_desc(const lpk_scene *s, int32_t r_idx, int32_t b_idx, uint64_t seed_base,
                               int32_t work_idx, lpk_band_desc *out);

/* Sink: called with each finished chunk, in order, on the calling thread.
 * Return 0 to continue, 1 to stop after this chunk (ControlFlow::Break,
 * src/pipeline.rs:984-989), negative to abort with LPK_EINVAL. */
typedef int32_t (*lpk_sink_fn)(void *user, const lpk_cf32 *chunk, int64_t n);

typedef struct lpk_band_result {
    int64_t n_samples;          /* samples handed to the sink */
    int32_t stopped_early;
    int32_t n_active;
    uint8_t unoccluded[256];    /* per active transmitter (pipeline.rs:905) */
} lpk_band_result;

/* generate_band flags. */
enum {
    LPK_NOISE_OFF = 0,          /* no AWGN (deterministic comparisons) */
    LPK_NOISE_ON = 1,           /* AWGN at the band's noise power */
    LPK_GEN_DEVICE_CLOCK = 2,   /* receiver clock on the GPU (white-FM walk counter-based and
                                   moment-matched, flicker track from the host stream) instead
                                   of the host stream; not for host-computed receiver positions */
    LPK_GEN_SPLIT = 4           /* split-precision fan-out (LPK_SOLVER_SPLIT) where the
                                   band allows it (stationary or orbiting receiver) */
};

/* generate_band (src/pipeline.rs:836-1019) on the GPU: the chunk loop with
 * the receiver's clock stream (host walk by default; on the device with
 * LPK_GEN_DEVICE_CLOCK; deterministic on the device when the clock has no
 * random part), the band-overlap gate, the fan-out kernel, AWGN and the rx
 * chain, handing each chunk to `sink`. `flags` is an OR of the values above. */
lpk_status lpk_generate_band(lpk_scene *s, int32_t r_idx, int32_t b_idx, uint64_t seed_base,
                             int32_t work_idx, int64_t chunk_samples, int32_t flags,
                             lpk_sink_fn sink, void *user, lpk_band_result *result);

/* Stream one band to <dir>/<name>.iq.c64 (raw little-endian complex64,
 * StreamingC64Writer, src/output/mod.rs:100-147). The JSON sidecar is
 * written by the caller, which holds the descriptor. */
lpk_status lpk_generate_band_to_file(lpk_scene *s, int32_t r_idx, int32_t b_idx, uint64_t seed_base,
                                     int32_t work_idx, int64_t chunk_samples, int32_t flags,
                                     const char *path, lpk_band_result *result);

/* Every work unit of the scene through one lpk_batch (run_scene_in_memory /
 * run_scene_to_dir, src/pipeline.rs:460-536, with the per-unit
 * generate_band calls fused): rounds of round_s seconds, each work unit's
 * chunk handed to sink(user, work_idx, chunk, n) in order. Work units whose
 * clock stays on the host stream (no LPK_GEN_DEVICE_CLOCK) or whose receiver
 * positions the host computes are rendered by lpk_generate_band instead,
 * after the batch. Flags as lpk_generate_band,
 * plus LPK_GEN_AUTOTUNE (tune the launch shape on the middle round first). */
enum { LPK_GEN_AUTOTUNE = 8 };
lpk_status lpk_generate_scene(lpk_scene *s, uint64_t seed_base, double round_s, int32_t flags,
                              lpk_unit_sink_fn sink, void *user);

/* run_scene_to_dir (src/pipeline.rs:494-536) through lpk_generate_scene:
 * work unit w's samples are appended to paths[w] (raw little-endian
 * complex64, StreamingC64Writer, src/output/mod.rs:100-147) from the pinned
 * staging while the next round renders. The JSON sidecars are written by
 * the caller, which holds the band metadata. */
lpk_status lpk_generate_scene_to_files(lpk_scene *s, uint64_t seed_base, double round_s, int32_t flags,
                                       const char *const *paths);

/* The flicker track of a receiver clock with a flicker floor, for the
 * device clock modes (lpk_band_desc.flicker_delta_s): out[m] = the flicker
 * Δt at m / 128 s after the band start, m = 0..n-1, the values the host
 * clock stream with the same spec and seed interpolates between
 * (Flicker::new and advance_to, src/clock/mod.rs:95-140; calibrated and
 * warmed on its own long-jumped copies of the clock's generator, so it does
 * not depend on the white-FM draws). seed: clock_seed(base, r_idx),
 * src/pipeline.rs:825-827. lpk_clock_flicker_len(duration_s) points cover a
 * band of duration_s. LPK_EINVAL for a spec without a flicker floor. */
int64_t lpk_clock_flicker_len(double duration_s);
lpk_status lpk_clock_flicker_table(const lpk_clock_cfg *spec, uint64_t seed, double *out, int64_t n);

/* Host clock stream (ClockStream, src/clock/mod.rs:229-347) exposed for
 * tests: delta_t_at over n monotone times. */
typedef struct lpk_clock lpk_clock;
lpk_status lpk_clock_new(const lpk_clock_cfg *spec, double start_epoch, double master_rate_hz,
                         uint64_t seed, lpk_clock **out);
lpk_status lpk_clock_delta_t(lpk_clock *c, const double *t, int64_t n, double *out);
void lpk_clock_free(lpk_clock *c);

#ifdef __cplusplus
}
#endif
#endif /* LIPIKA_CUDA_H */
