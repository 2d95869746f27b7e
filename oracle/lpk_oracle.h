/*
 * lpk_oracle.h — CPU ORACLE for the lipika IQ-generation hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates the reference's Rust
 * algorithm in plain C so that the CUDA backend can be checked against it.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it, and only as the checker or the timed CPU baseline; the product
 * (lipika_b200/, liblipika_cuda.so) never links or calls it.
 *
 * Parity pins: every function cites the reference file:line it restates and
 * is checked against the reference's own known-answer tests
 * (tests/test_oracle_known_answers.py). Third-party RNG streams (rand 0.8
 * gen_bool / gen_range, rand_xoshiro 0.6 seeding, rand_distr 0.4 Normal) are
 * restated from their published algorithms; agreement with those crates is
 * UNPINNED (no crate source or golden vector exists in the reference), and
 * the Normal sampler is a documented Box–Muller, not rand_distr's ziggurat.
 */
#ifndef LPK_ORACLE_H
#define LPK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/lipika_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- RNG (published algorithms) ---------------- */
typedef struct { uint64_t s[4]; } orc_xoshiro;
void orc_xoshiro_seed(orc_xoshiro *r, uint64_t seed);          /* SplitMix64 fill */
uint64_t orc_xoshiro_next(orc_xoshiro *r);                      /* xoshiro256++ */
void orc_xoshiro_long_jump(orc_xoshiro *r);
int orc_gen_bool_half(orc_xoshiro *r);                          /* rand 0.8 Bernoulli(0.5) */
uint32_t orc_gen_range_u8_16(orc_xoshiro *r);                   /* rand 0.8 gen_range(0..16u8) */
double orc_std_normal(orc_xoshiro *r);                          /* Box–Muller, 2 draws */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Counter-based AWGN pair of the CUDA backend's noise spec (re, im). */
void orc_noise_pair(uint64_t seed, int64_t global_index, float *z_re, float *z_im);

/* ---------------- geometry ---------------- */
void orc_geodetic_to_ecef(double lat_deg, double lon_deg, double h_m, double out[3]);
void orc_kepler_position_ecef(const lpk_trajectory_cfg *k, double t_unix, double out[3]);

enum { ORC_TRAJ_STATIONARY = 0, ORC_TRAJ_PRECOMPUTED = 1, ORC_TRAJ_RAW = 2 };
typedef struct orc_traj {
    int32_t kind;
    int32_t reserved;
    int64_t n;               /* grid points */
    double pos[3];           /* stationary */
    double t0_unix, dt_s;    /* precomputed grid */
    double *grid;            /* (3, n) axis-major, as ndarray stores it */
    double max_speed_m_s, max_radius_m;
    lpk_trajectory_cfg raw;  /* raw (receiver) trajectory */
} orc_traj;

int orc_traj_sample(const lpk_trajectory_cfg *cfg, double t0_unix, double duration_s,
                    double grid_dt_s, orc_traj *out);
int orc_traj_for_transmitter(const lpk_trajectory_cfg *cfg, double scene_epoch,
                             double duration_s, orc_traj *out);
int orc_traj_for_receiver(const lpk_trajectory_cfg *cfg, double scene_epoch, orc_traj *out);
void orc_traj_position(const orc_traj *t, double t_unix, double out[3]);
void orc_traj_position_batch(const orc_traj *t, const double *t_unix, int64_t n, double *out3n);
void orc_traj_free(orc_traj *t);

/* ---------------- signals ---------------- */
int orc_elapsed_periods(double elapsed_s, double rate_hz, int64_t *whole, double *frac);
int orc_frame_anchor(double render_epoch, double signal_epoch, double rate_hz, int64_t n_symbols,
                     double *epoch_rel_s, int64_t *symbol_offset);
int orc_cw_anchor_phase(double render_epoch, double signal_epoch, double f_hz, double *phase);
void orc_ca_code(int prn, int8_t out[1023]);
int8_t orc_nav_bit_pm(uint64_t seed, int64_t bit_idx);
int orc_frame_index(int64_t raw, int64_t n, int has_repeat, int64_t repeat_from, int64_t *idx);

typedef struct orc_signal {
    int32_t kind;            /* LPK_SIG_* */
    int32_t nav;             /* ca: LPK_NAV_* */
    double carrier_hz;
    double epoch_rel_s;
    double rate_hz;
    int32_t has_repeat;
    int32_t cw_anchored;
    int64_t repeat_from;
    int64_t n;               /* frame length (bits / symbols) */
    int8_t *pm;              /* bpsk ±1 */
    uint8_t *bits;           /* ook 0/1 */
    float *sym;              /* qam16 (re, im) pairs */
    int8_t code[1023];       /* ca chips ±1 */
    uint64_t nav_seed;       /* dummy nav folded seed */
    int8_t *nav_bits;        /* full nav table */
    int64_t nav_n;
    double cw_offset_hz;
    double cw_phase0;
    int32_t has_gate;
    int32_t gate_n;
    double gate_period_s, gate_phase_s;
    double *gate_on;         /* gate_n (start, end) pairs */
} orc_signal;

int orc_signal_build(const lpk_transmitter_cfg *cfg, const lpk_scene_cfg *scene, orc_signal *out);
void orc_signal_eval(const orc_signal *s, const double *t_emit, int64_t n, float *out2n);
int orc_gate_is_on(const orc_signal *s, double t);
void orc_signal_free(orc_signal *s);

/* ---------------- channel ---------------- */
typedef struct orc_antenna {
    double peak_dbi, horizon_dbi, fb_db, cutoff_deg;
    int32_t has_cutoff;
    int32_t reserved;
} orc_antenna;
float orc_antenna_amplitude(const orc_antenna *a, double elev_deg);

void orc_solve_emission_times(const orc_traj *src, const double *obs3n, const double *t_rel_utc,
                              int64_t n, double epoch, int iterations,
                              double *t_emit, double *ranges);
/* Fixed point iterated until |dt| <= tol_s (long double arithmetic): the
 * converged truth the 2-iteration reference result is compared with. */
void orc_solve_converged(const orc_traj *src, const double *obs3n, const double *t_rel_utc,
                         int64_t n, double epoch, double tol_s, int max_iter,
                         double *t_emit, double *ranges, int32_t *iters_used);
int orc_accumulate(float *acc2n, const orc_signal *sig, const orc_traj *traj, const double *obs3n,
                   const double *t_local, const double *t_utc, const double *delta_t, int64_t n,
                   double lo_hz, double tx_power_w, double epoch, int iterations,
                   const orc_antenna *antenna);
double orc_thermal_noise_power_w(double temperature_k, double bandwidth_hz);
int orc_bands_overlap(double tx_carrier, double tx_bw, double band_lo, double band_bw);

/* ---------------- rx chain ---------------- */
enum { ORC_POST_GAIN = 0, ORC_POST_NONLIN = 1, ORC_POST_ADC = 2 };
typedef struct orc_post_op { int32_t kind; uint32_t bits; double a; } orc_post_op;
typedef struct orc_rx_chain {
    int32_t has_antenna;
    int32_t n_post;
    orc_antenna antenna;
    orc_post_op post[3];
} orc_rx_chain;
void orc_rx_chain_from_config(const lpk_frontend_cfg *fe, int has_frontend, orc_rx_chain *out);
void orc_rx_apply_post_sum(const orc_rx_chain *c, float *iq2n, int64_t n);
/* ADC codes round(clamp(x)/lsb) of the chain's last ADC stage (0 if none). */
int orc_adc_codes(const orc_rx_chain *c, const float *iq2n, int64_t n, int32_t *codes2n);

/* ---------------- clock ---------------- */
typedef struct orc_clock orc_clock;
orc_clock *orc_clock_new(const lpk_clock_cfg *spec, double start_epoch, double master_rate_hz,
                         uint64_t seed);
double orc_clock_delta_t_at(orc_clock *c, double t);
double orc_clock_delta_t_at_master_index(orc_clock *c, int64_t k);
void orc_clock_free(orc_clock *c);
uint64_t orc_clock_seed(uint64_t base, uint64_t r_idx);
uint64_t orc_noise_seed(uint64_t base, uint64_t work_idx);

/* ---------------- scene / band loop ---------------- */
typedef struct orc_scene orc_scene;
int orc_scene_prepare(const lpk_scene_cfg *cfg, orc_scene **out);
void orc_scene_free(orc_scene *s);
int orc_scene_n_work(const orc_scene *s);
int orc_scene_work(const orc_scene *s, int work_idx, int *r_idx, int *b_idx);
int64_t orc_band_n_samples(const orc_scene *s, int r_idx, int b_idx);
int orc_band_active(const orc_scene *s, int r_idx, int b_idx, int32_t *active, int cap);
const orc_signal *orc_scene_signal(const orc_scene *s, int tx);
const orc_traj *orc_scene_traj(const orc_scene *s, int tx);
double orc_scene_tx_power_w(const orc_scene *s, int tx);

/* noise_mode: 0 = none, 1 = counter-based spec of the CUDA backend,
 *             2 = sequential xoshiro stream (the reference's structure). */
enum { ORC_NOISE_NONE = 0, ORC_NOISE_COUNTER = 1, ORC_NOISE_SEQUENTIAL = 2 };
int orc_generate_band(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int work_idx,
                      int64_t chunk_samples, int n_threads, int noise_mode,
                      int64_t sample_limit, float *out_iq2n, double *out_delta,
                      uint8_t *unoccluded);
int orc_generate_band_window(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int work_idx,
                             int64_t chunk_samples, int n_threads, int noise_mode, int64_t sample_start,
                             int64_t sample_limit, float *out, double *out_delta, uint8_t *unoccluded);
/* Single-thread cost of each section of the loop on the first n samples of
 * a band (ns per band or tx-rx sample; see lpk_oracle.c). */
int orc_profile_sections(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int64_t n, double *ns_out);

#ifdef __cplusplus
}
#endif
#endif
