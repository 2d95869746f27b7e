/*
 * lpk_oracle.c — CPU ORACLE (test infrastructure only; see lpk_oracle.h).
 *
 * A plain-C restatement of the reference's IQ-generation path. Built with
 * -O2 -ffp-contract=off and glibc libm, which is what the reference's Rust
 * f64/f32 arithmetic and sin/cos/asin/pow calls resolve to on x86_64 Linux,
 * so every f64 operation here is performed in the reference's order with the
 * reference's rounding. Each function cites the reference file:line it
 * restates.
 */
#include "lpk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#define TAU 6.283185307179586476925286766559
static const double SPEED_OF_LIGHT_M_S = 299792458.0;      /* src/lib.rs:53 */
static const double EMISSION_INITIAL_LAG_S = 0.07;        /* src/channel/mod.rs:23 */
static const double EARTH_ROTATION_RATE = 7.2921151467e-5; /* src/channel/mod.rs:27 */
static const double GM_EARTH = 3.986005e14;               /* src/geometry/kepler.rs:12 */
static const double BOLTZMANN = 1.380649e-23;             /* src/channel/mod.rs:301 */
static const double CA_CHIP_RATE_HZ = 1023000.0;          /* src/signal/ca_code.rs:23 */
static const double NAV_BIT_RATE_HZ = 50.0;               /* src/signal/ca_code.rs:27 */
static const double GRID_DT_S = 0.01;                     /* src/pipeline.rs:62 */
static const int NEWTON_ITERATIONS = 2;                   /* src/pipeline.rs:56 */

/* Rust f64::to_radians / to_degrees (core::f64). */
static double to_radians(double x) { return x * (M_PI / 180.0); }
static double to_degrees(double x) { return x * 57.2957795130823208767981548141051703; }

/* Rust `f64 as i64` saturates and maps NaN to 0. */
static int64_t f64_to_i64(double x) {
    if (x != x) return 0;
    if (x >= 9223372036854775807.0) return INT64_MAX;
    if (x <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)x;
}
static int64_t i64_rem_euclid(int64_t a, int64_t b) {
    int64_t r = a % b;
    if (r < 0) r = (b < 0) ? r - b : r + b;
    return r;
}
static double f64_rem_euclid(double a, double b) {
    double r = fmod(a, b);
    return (r < 0.0) ? r + fabs(b) : r;
}
static double f64_clamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
static float f32_clamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

/* ======================= RNG ======================= */
static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t splitmix64_next(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* rand_xoshiro 0.6 Xoshiro256PlusPlus::seed_from_u64: the 256-bit state is
 * filled from a SplitMix64 stream seeded with `seed` (used at
 * src/pipeline.rs:165, :180, :194, :871, :873). */
void orc_xoshiro_seed(orc_xoshiro *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64_next(&x);
}

/* xoshiro256++ (Blackman & Vigna), next_u64. */
uint64_t orc_xoshiro_next(orc_xoshiro *r) {
    uint64_t *s = r->s;
    uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

/* xoshiro256 long_jump (2^192 steps), used by the flicker generator
 * (src/clock/mod.rs:102, :120-121). */
void orc_xoshiro_long_jump(orc_xoshiro *r) {
    static const uint64_t LJ[4] = {0x76e15d3efefdcbbfULL, 0xc5004e441c522fb3ULL,
                                   0x77710069854ee241ULL, 0x39109bb02acbe635ULL};
    uint64_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = 0; i < 4; i++)
        for (int b = 0; b < 64; b++) {
            if (LJ[i] & (1ULL << b)) {
                s0 ^= r->s[0]; s1 ^= r->s[1]; s2 ^= r->s[2]; s3 ^= r->s[3];
            }
            orc_xoshiro_next(r);
        }
    r->s[0] = s0; r->s[1] = s1; r->s[2] = s2; r->s[3] = s3;
}

/* rand 0.8 `gen_bool(0.5)`: Bernoulli with p_int = 0.5 * 2^64 = 2^63;
 * true iff the next u64 is below it (src/signal/bpsk.rs:39, ook.rs:41). */
int orc_gen_bool_half(orc_xoshiro *r) { return orc_xoshiro_next(r) < 0x8000000000000000ULL; }

/* rand 0.8 `gen_range(0..16)` for u8 (src/signal/qam16.rs:76): widening
 * multiply of a u32 draw (the upper half of next_u64) by the range 16; with
 * a power-of-two range nothing is rejected, so the value is v >> 28. */
uint32_t orc_gen_range_u8_16(orc_xoshiro *r) {
    uint32_t v = (uint32_t)(orc_xoshiro_next(r) >> 32);
    return (uint32_t)(((uint64_t)v * 16ULL) >> 32);
}

/* Standard normal by Box–Muller from two 53-bit uniforms. The reference
 * uses rand_distr's ziggurat (src/clock/mod.rs:190, channel/mod.rs:329);
 * its stream is not reproduced, only its distribution. The product host
 * uses this same documented sampler, so host-fed clock walks agree. */
double orc_std_normal(orc_xoshiro *r) {
    double u1 = (double)((orc_xoshiro_next(r) >> 11) + 1) * 0x1.0p-53; /* (0, 1] */
    double u2 = (double)(orc_xoshiro_next(r) >> 11) * 0x1.0p-53;       /* [0, 1) */
    return sqrt(-2.0 * log(u1)) * cos(TAU * u2);
}

/* Philox4x32-10 (Salmon et al., SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; round++) {
        if (round > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* The CUDA backend's AWGN spec: one Philox block per (noise seed, pair of
 * global band-sample indices 2p, 2p+1); words 0-1 drive sample 2p and
 * words 2-3 sample 2p+1, each through Box–Muller in f32. */
void orc_noise_pair(uint64_t seed, int64_t g, float *z_re, float *z_im) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint64_t p = (uint64_t)g >> 1;
    uint32_t ctr[4] = {(uint32_t)p, (uint32_t)(p >> 32), 0x4E4F4953u, 0u};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    int h = (int)(g & 1) * 2;
    float u1 = ((float)(x[h] >> 8) + 1.0f) * 0x1.0p-24f;
    float u2 = (float)(x[h + 1] >> 8) * 0x1.0p-24f;
    float rr = sqrtf(-2.0f * logf(u1));
    float ang = 6.28318548f * u2 - 3.14159274f;  /* the device takes sin/cos on [-pi, pi) */
    *z_re = rr * cosf(ang);
    *z_im = rr * sinf(ang);
}

/* ======================= geometry ======================= */
/* src/geometry/ecef.rs:3-20 */
void orc_geodetic_to_ecef(double lat_deg, double lon_deg, double h_m, double out[3]) {
    const double A = 6378137.0;
    const double F = 1.0 / 298.257223563;
    const double E2 = F * (2.0 - F);
    double lat = to_radians(lat_deg);
    double lon = to_radians(lon_deg);
    double sin_lat = sin(lat);
    double cos_lat = cos(lat);
    double n = A / sqrt(1.0 - E2 * sin_lat * sin_lat);
    out[0] = (n + h_m) * cos_lat * cos(lon);
    out[1] = (n + h_m) * cos_lat * sin(lon);
    out[2] = (n * (1.0 - E2) + h_m) * sin_lat;
}

/* src/geometry/kepler.rs:27-85 (position only). */
void orc_kepler_position_ecef(const lpk_trajectory_cfg *k, double t_unix, double out[3]) {
    double r = k->semi_major_axis_m;
    double a3 = r * r * r; /* powi(3) */
    double n = sqrt(GM_EARTH / a3);
    double dt = t_unix - k->epoch_unix;
    double nu = to_radians(k->true_anomaly_deg_at_epoch) + n * dt;
    double s_nu = sin(nu), c_nu = cos(nu);
    double incl = to_radians(k->inclination_deg);
    double s_i = sin(incl), c_i = cos(incl);
    double raan = to_radians(k->raan_deg);
    double s_o = sin(raan), c_o = cos(raan);
    double xp = r * c_nu;
    double yp = r * s_nu;
    double y1 = yp * c_i;
    double z1 = yp * s_i;
    double x_eci = xp * c_o - y1 * s_o;
    double y_eci = xp * s_o + y1 * c_o;
    double z_eci = z1;
    double theta = EARTH_ROTATION_RATE * (t_unix - k->epoch_unix);
    double s = sin(theta), c = cos(theta);
    out[0] = x_eci * c + y_eci * s;
    out[1] = -x_eci * s + y_eci * c;
    out[2] = z_eci;
}

static int raw_position(const lpk_trajectory_cfg *cfg, double t_unix, double out[3]) {
    switch (cfg->kind) {
    case LPK_TRAJ_STATIONARY_GEODETIC:
        orc_geodetic_to_ecef(cfg->lat_deg, cfg->lon_deg, cfg->h_m, out);
        return 0;
    case LPK_TRAJ_STATIONARY_ECEF:
        out[0] = cfg->x_m; out[1] = cfg->y_m; out[2] = cfg->z_m;
        return 0;
    case LPK_TRAJ_CIRCULAR_KEPLERIAN:
        orc_kepler_position_ecef(cfg, t_unix, out);
        return 0;
    default:
        return -1;
    }
}

/* src/geometry/precomputed.rs:220-241 */
static void path_bounds(const double *g, int64_t n, double dt, double *vmax, double *rmax) {
    double max_seg2 = 0.0, max_r2 = 0.0;
    int finite = 1;
    for (int64_t k = 0; k < n; k++) {
        double p0 = g[k], p1 = g[n + k], p2 = g[2 * n + k];
        double r2 = p0 * p0 + p1 * p1 + p2 * p2;
        finite &= isfinite(r2);
        if (r2 > max_r2) max_r2 = r2;
        if (k + 1 < n) {
            double d0 = g[k + 1] - p0, d1 = g[n + k + 1] - p1, d2 = g[2 * n + k + 1] - p2;
            double seg2 = d0 * d0 + d1 * d1 + d2 * d2;
            finite &= isfinite(seg2);
            if (seg2 > max_seg2) max_seg2 = seg2;
        }
    }
    if (finite) { *vmax = sqrt(max_seg2) / dt; *rmax = sqrt(max_r2); }
    else { *vmax = NAN; *rmax = NAN; }
}

/* PrecomputedTrajectory::sample, src/geometry/precomputed.rs:180-204 */
int orc_traj_sample(const lpk_trajectory_cfg *cfg, double t0_unix, double duration_s,
                    double grid_dt_s, orc_traj *out) {
    memset(out, 0, sizeof *out);
    if (!(grid_dt_s > 0.0)) return -1;
    const double pad_s = 0.5;
    double start = t0_unix - pad_s;
    double total = duration_s + 2.0 * pad_s;
    int64_t n = (int64_t)ceil(total / grid_dt_s) + 1;
    if (n < 2) return -1;
    out->kind = ORC_TRAJ_PRECOMPUTED;
    out->n = n;
    out->t0_unix = start;
    out->dt_s = grid_dt_s;
    out->grid = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    if (!out->grid) return -2;
    for (int64_t i = 0; i < n; i++) {
        double p[3];
        if (raw_position(cfg, start + (double)i * grid_dt_s, p)) return -1;
        out->grid[i] = p[0];
        out->grid[n + i] = p[1];
        out->grid[2 * n + i] = p[2];
    }
    path_bounds(out->grid, n, grid_dt_s, &out->max_speed_m_s, &out->max_radius_m);
    return 0;
}

/* Transmitter::from_config, src/pipeline.rs:316-333: stationary kinds are
 * evaluated once at the scene epoch, everything else is tabulated. */
int orc_traj_for_transmitter(const lpk_trajectory_cfg *cfg, double scene_epoch,
                             double duration_s, orc_traj *out) {
    memset(out, 0, sizeof *out);
    if (cfg->kind == LPK_TRAJ_STATIONARY_GEODETIC || cfg->kind == LPK_TRAJ_STATIONARY_ECEF) {
        out->kind = ORC_TRAJ_STATIONARY;
        return raw_position(cfg, scene_epoch, out->pos);
    }
    if (cfg->kind != LPK_TRAJ_CIRCULAR_KEPLERIAN) return -3;
    return orc_traj_sample(cfg, scene_epoch, duration_s, GRID_DT_S, out);
}

/* Receiver::from_config, src/pipeline.rs:352-363: the raw trajectory. */
int orc_traj_for_receiver(const lpk_trajectory_cfg *cfg, double scene_epoch, orc_traj *out) {
    memset(out, 0, sizeof *out);
    if (cfg->kind == LPK_TRAJ_STATIONARY_GEODETIC || cfg->kind == LPK_TRAJ_STATIONARY_ECEF) {
        out->kind = ORC_TRAJ_STATIONARY;
        return raw_position(cfg, scene_epoch, out->pos);
    }
    if (cfg->kind != LPK_TRAJ_CIRCULAR_KEPLERIAN) return -3;
    out->kind = ORC_TRAJ_RAW;
    out->raw = *cfg;
    return 0;
}

/* PrecomputedTrajectory::position_ecef, src/geometry/precomputed.rs:111-121 */
void orc_traj_position(const orc_traj *t, double t_unix, double out[3]) {
    if (t->kind == ORC_TRAJ_STATIONARY) {
        out[0] = t->pos[0]; out[1] = t->pos[1]; out[2] = t->pos[2];
        return;
    }
    if (t->kind == ORC_TRAJ_RAW) { raw_position(&t->raw, t_unix, out); return; }
    double f = (t_unix - t->t0_unix) / t->dt_s;
    int64_t lo = f64_to_i64(floor(f));
    if (lo < 0) lo = 0;
    if (lo > t->n - 2) lo = t->n - 2;
    double frac = f64_clamp(f - (double)lo, 0.0, 1.0);
    const double *a = t->grid;
    int64_t n = t->n;
    out[0] = a[lo] * (1.0 - frac) + a[lo + 1] * frac;
    out[1] = a[n + lo] * (1.0 - frac) + a[n + lo + 1] * frac;
    out[2] = a[2 * n + lo] * (1.0 - frac) + a[2 * n + lo + 1] * frac;
}

/* position_ecef_batch: src/geometry/precomputed.rs:136-153 (multiplies by a
 * precomputed 1/dt, unlike the single query), stationary.rs:30-39,
 * kepler.rs:92-102. Output (3, n) axis-major. */
void orc_traj_position_batch(const orc_traj *t, const double *tu, int64_t m, double *out) {
    if (t->kind == ORC_TRAJ_PRECOMPUTED) {
        double inv_dt = 1.0 / t->dt_s;
        int64_t max_lo = t->n - 2;
        const double *a = t->grid;
        int64_t n = t->n;
        for (int64_t i = 0; i < m; i++) {
            double f = (tu[i] - t->t0_unix) * inv_dt;
            int64_t lo = f64_to_i64(floor(f));
            if (lo < 0) lo = 0;
            if (lo > max_lo) lo = max_lo;
            double frac = f64_clamp(f - (double)lo, 0.0, 1.0);
            double omf = 1.0 - frac;
            out[i] = a[lo] * omf + a[lo + 1] * frac;
            out[m + i] = a[n + lo] * omf + a[n + lo + 1] * frac;
            out[2 * m + i] = a[2 * n + lo] * omf + a[2 * n + lo + 1] * frac;
        }
        return;
    }
    for (int64_t i = 0; i < m; i++) {
        double p[3];
        orc_traj_position(t, tu[i], p);
        out[i] = p[0]; out[m + i] = p[1]; out[2 * m + i] = p[2];
    }
}

void orc_traj_free(orc_traj *t) { free(t->grid); t->grid = NULL; }

/* ======================= signals ======================= */
/* src/signal/mod.rs:49-69 */
int orc_elapsed_periods(double elapsed_s, double rate_hz, int64_t *whole_out, double *frac_out) {
    double p = elapsed_s * rate_hz;
    if (!isfinite(p) || fabs(p) >= 9.0e18) return -1;
    double err = fma(elapsed_s, rate_hz, -p);
    double whole = floor(p);
    double frac = (p - whole) + err;
    if (frac < 0.0) { whole -= 1.0; frac += 1.0; }
    else if (frac >= 1.0) { whole += 1.0; frac -= 1.0; }
    *whole_out = (int64_t)whole;
    *frac_out = frac;
    return 0;
}

/* FrameAnchor::at, src/signal/mod.rs:86-101 */
int orc_frame_anchor(double render_epoch, double signal_epoch, double rate_hz, int64_t n_symbols,
                     double *epoch_rel_s, int64_t *symbol_offset) {
    if (!(rate_hz > 0.0)) return -1;
    int64_t whole;
    double frac;
    if (orc_elapsed_periods(render_epoch - signal_epoch, rate_hz, &whole, &frac)) return -1;
    *epoch_rel_s = -frac / rate_hz;
    *symbol_offset = i64_rem_euclid(whole, n_symbols > 1 ? n_symbols : 1);
    return 0;
}

/* ContinuousWave::anchor_phase, src/signal/cw.rs:22-34 */
int orc_cw_anchor_phase(double render_epoch, double signal_epoch, double f_hz, double *phase) {
    int64_t whole;
    double frac;
    if (orc_elapsed_periods(render_epoch - signal_epoch, f_hz, &whole, &frac)) return -1;
    *phase = TAU * frac;
    return 0;
}

/* src/signal/ca_code.rs:34-78 (G1/G2 LFSRs, IS-GPS-200 taps). */
void orc_ca_code(int prn, int8_t out[1023]) {
    static const int TAPS[32][2] = {
        {2, 6}, {3, 7}, {4, 8}, {5, 9}, {1, 9}, {2, 10}, {1, 8}, {2, 9}, {3, 10},
        {2, 3}, {3, 4}, {5, 6}, {6, 7}, {7, 8}, {8, 9}, {9, 10}, {1, 4}, {2, 5},
        {3, 6}, {4, 7}, {5, 8}, {6, 9}, {1, 3}, {4, 6}, {5, 7}, {6, 8}, {7, 9},
        {8, 10}, {1, 6}, {2, 7}, {3, 8}, {4, 9}};
    int8_t g1[10], g2[10];
    for (int i = 0; i < 10; i++) { g1[i] = 1; g2[i] = 1; }
    int ta = TAPS[prn - 1][0] - 1, tb = TAPS[prn - 1][1] - 1;
    for (int k = 0; k < 1023; k++) {
        int8_t o1 = g1[9];
        int8_t o2 = g2[ta] ^ g2[tb];
        int8_t f1 = g1[2] ^ g1[9];
        int8_t f2 = g2[1] ^ g2[2] ^ g2[5] ^ g2[7] ^ g2[8] ^ g2[9];
        for (int i = 9; i > 0; i--) { g1[i] = g1[i - 1]; g2[i] = g2[i - 1]; }
        g1[0] = f1;
        g2[0] = f2;
        out[k] = (int8_t)(1 - 2 * (o1 ^ o2));
    }
}

/* NavData::bit_pm, src/signal/ca_code.rs:94-108 */
int8_t orc_nav_bit_pm(uint64_t seed, int64_t bit_idx) {
    static const uint8_t PRE[8] = {1, 0, 0, 0, 1, 0, 1, 1};
    int64_t pos = i64_rem_euclid(bit_idx, 300);
    uint8_t bit;
    if (pos < 8) {
        bit = PRE[pos];
    } else {
        uint64_t x = seed ^ ((uint64_t)bit_idx * 0x9E3779B97F4A7C15ULL);
        x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ULL;
        x ^= x >> 27; x *= 0x94D049BB133111EBULL;
        x ^= x >> 31;
        bit = (uint8_t)(x & 1);
    }
    return (int8_t)(1 - 2 * (int)bit);
}

/* frame_index, src/signal/mod.rs:108-115. Returns 1 and sets *idx when the
 * raw count maps to a frame symbol, 0 when the frame is silent there. */
int orc_frame_index(int64_t raw, int64_t n, int has_repeat, int64_t k, int64_t *idx) {
    if (!has_repeat) {
        if (raw >= 0 && raw < n) { *idx = raw; return 1; }
        return 0;
    }
    if (n <= 0) return 0;
    *idx = i64_rem_euclid((int64_t)((uint64_t)raw + (uint64_t)k), n);
    return 1;
}

static float gray_level(uint8_t b0, uint8_t b1) { /* src/signal/qam16.rs:20-27 */
    if (b0 == 0 && b1 == 0) return -3.0f;
    if (b0 == 0 && b1 == 1) return -1.0f;
    if (b0 == 1 && b1 == 1) return 1.0f;
    return 3.0f;
}
static void map_symbol(const uint8_t b[4], float *re, float *im) { /* qam16.rs:32-34 */
    const float S = 0.31622777f;
    *re = gray_level(b[0], b[1]) * S;
    *im = gray_level(b[2], b[3]) * S;
}

/* build_signal, src/pipeline.rs:141-253 (LNAV "full" is out of scope). */
int orc_signal_build(const lpk_transmitter_cfg *cfg, const lpk_scene_cfg *scene, orc_signal *s) {
    memset(s, 0, sizeof *s);
    double render_epoch = scene->epoch_unix;
    int anchored = 0;
    double anchor_epoch = 0.0;
    if (cfg->has_signal_epoch) { anchored = 1; anchor_epoch = cfg->signal_epoch_unix; }
    else if (scene->time_base == LPK_TIME_BASE_ABSOLUTE) {
        anchored = 1;
        anchor_epoch = scene->default_signal_epoch_unix;
    }
    s->kind = cfg->kind;
    s->carrier_hz = cfg->carrier_hz;
    orc_xoshiro rng;
    switch (cfg->kind) {
    case LPK_SIG_CW:
        s->cw_offset_hz = cfg->baseband_offset_hz;
        if (anchored) {
            s->cw_anchored = 1;
            if (orc_cw_anchor_phase(render_epoch, anchor_epoch, cfg->baseband_offset_hz, &s->cw_phase0))
                return -1;
        }
        break;
    case LPK_SIG_BPSK:
    case LPK_SIG_OOK:
    case LPK_SIG_QAM16: {
        orc_xoshiro_seed(&rng, cfg->payload_seed);
        s->rate_hz = cfg->rate_hz;
        s->epoch_rel_s = 0.0;
        if (cfg->kind == LPK_SIG_BPSK) {
            s->n = cfg->sync_n + cfg->payload_n;
            s->pm = (int8_t *)malloc((size_t)(s->n ? s->n : 1));
            for (int i = 0; i < cfg->sync_n; i++) s->pm[i] = cfg->sync_word[i];
            for (int64_t i = 0; i < cfg->payload_n; i++)
                s->pm[cfg->sync_n + i] = orc_gen_bool_half(&rng) ? 1 : -1;
        } else if (cfg->kind == LPK_SIG_OOK) {
            for (int i = 0; i < cfg->sync_n; i++)
                if (cfg->sync_word[i] < 0 || cfg->sync_word[i] > 1) return -1;
            s->n = cfg->sync_n + cfg->payload_n;
            s->bits = (uint8_t *)malloc((size_t)(s->n ? s->n : 1));
            for (int i = 0; i < cfg->sync_n; i++) s->bits[i] = (uint8_t)cfg->sync_word[i];
            for (int64_t i = 0; i < cfg->payload_n; i++)
                s->bits[cfg->sync_n + i] = (uint8_t)orc_gen_bool_half(&rng);
        } else {
            for (int i = 0; i < cfg->sync_n; i++)
                if (cfg->sync_word[i] < 0 || cfg->sync_word[i] > 1) return -1;
            if (cfg->sync_n % 4) return -1;
            int64_t ns = cfg->sync_n / 4;
            s->n = ns + cfg->payload_n;
            s->sym = (float *)malloc(sizeof(float) * 2 * (size_t)(s->n ? s->n : 1));
            for (int64_t i = 0; i < ns; i++) {
                uint8_t b[4];
                for (int j = 0; j < 4; j++) b[j] = (uint8_t)cfg->sync_word[4 * i + j];
                map_symbol(b, &s->sym[2 * i], &s->sym[2 * i + 1]);
            }
            for (int64_t i = 0; i < cfg->payload_n; i++) {
                uint32_t v = orc_gen_range_u8_16(&rng);
                uint8_t b[4] = {(uint8_t)((v >> 3) & 1), (uint8_t)((v >> 2) & 1),
                                (uint8_t)((v >> 1) & 1), (uint8_t)(v & 1)};
                map_symbol(b, &s->sym[2 * (ns + i)], &s->sym[2 * (ns + i) + 1]);
            }
        }
        if (anchored) {
            s->has_repeat = 1;
            if (orc_frame_anchor(render_epoch, anchor_epoch, cfg->rate_hz, s->n, &s->epoch_rel_s,
                                 &s->repeat_from))
                return -1;
        }
        break;
    }
    case LPK_SIG_CA_CODE:
        if (cfg->prn < 1 || cfg->prn > 32) return -1;
        orc_ca_code(cfg->prn, s->code);
        if (scene->time_base == LPK_TIME_BASE_SCENE) {
            s->epoch_rel_s = cfg->ca_epoch_unix - render_epoch;
            if (cfg->nav == LPK_NAV_OFF) s->nav = LPK_NAV_OFF;
            else if (cfg->nav == LPK_NAV_DUMMY) {
                s->nav = LPK_NAV_DUMMY;
                s->nav_seed = cfg->nav_seed + (uint64_t)cfg->prn * 0xD1B54A32D192ED03ULL;
            } else return -3; /* LNAV generation is not restated */
        } else {
            if (cfg->nav != LPK_NAV_OFF) return -1;
            double epoch_rel;
            int64_t off;
            if (orc_frame_anchor(render_epoch, cfg->ca_epoch_unix, CA_CHIP_RATE_HZ / 1023.0, 1,
                                 &epoch_rel, &off))
                return -1;
            s->epoch_rel_s = epoch_rel;
            s->nav = LPK_NAV_OFF;
        }
        break;
    default:
        return -1;
    }
    if (cfg->has_gate) { /* BurstGate::anchored / new, src/signal/gate.rs:36-55 */
        double period = cfg->gate_period_s;
        if (!(period > 0.0) || !isfinite(period)) return -1;
        s->has_gate = 1;
        s->gate_n = cfg->gate_n_bursts;
        s->gate_on = (double *)malloc(sizeof(double) * 2 * (size_t)(s->gate_n ? s->gate_n : 1));
        for (int i = 0; i < s->gate_n; i++) {
            double off = cfg->gate_bursts[2 * i], dur = cfg->gate_bursts[2 * i + 1];
            if (!(off >= 0.0) || !(dur > 0.0) || !(off + dur <= period)) return -1;
            s->gate_on[2 * i] = off;
            s->gate_on[2 * i + 1] = off + dur;
        }
        double phase = render_epoch - cfg->gate_epoch_unix;
        if (!isfinite(phase)) return -1;
        s->gate_period_s = period;
        s->gate_phase_s = f64_rem_euclid(phase, period);
    }
    return 0;
}

/* BurstGate::is_on, src/signal/gate.rs:71-77 */
int orc_gate_is_on(const orc_signal *s, double t) {
    double u = f64_rem_euclid(t + s->gate_phase_s, s->gate_period_s);
    if (u >= s->gate_period_s) u = 0.0;
    for (int i = 0; i < s->gate_n; i++)
        if (u >= s->gate_on[2 * i] && u < s->gate_on[2 * i + 1]) return 1;
    return 0;
}

/* evaluate_baseband_batch of cw.rs:41-52, bpsk.rs:58-71, ook.rs:60-74,
 * qam16.rs:96-109, ca_code.rs:167-193, wrapped by gate.rs:91-105. */
void orc_signal_eval(const orc_signal *s, const double *t_emit, int64_t n, float *out) {
    for (int64_t i = 0; i < n; i++) {
        double t = t_emit[i];
        float re = 0.0f, im = 0.0f;
        switch (s->kind) {
        case LPK_SIG_CW: {
            double omega = TAU * s->cw_offset_hz;
            float ph = s->cw_anchored ? (float)f64_rem_euclid(omega * t + s->cw_phase0, TAU)
                                      : (float)(omega * t);
            re = cosf(ph);
            im = sinf(ph);
            break;
        }
        case LPK_SIG_BPSK:
        case LPK_SIG_OOK:
        case LPK_SIG_QAM16: {
            double f = (t - s->epoch_rel_s) * s->rate_hz;
            int64_t raw = f64_to_i64(floor(f)), k;
            if (orc_frame_index(raw, s->n, s->has_repeat, s->repeat_from, &k)) {
                if (s->kind == LPK_SIG_BPSK) re = (float)s->pm[k];
                else if (s->kind == LPK_SIG_OOK) re = (float)s->bits[k];
                else { re = s->sym[2 * k]; im = s->sym[2 * k + 1]; }
            }
            break;
        }
        case LPK_SIG_CA_CODE: {
            double dt = t - s->epoch_rel_s;
            double chip_phase = dt * CA_CHIP_RATE_HZ;
            int64_t idx = f64_to_i64(floor(chip_phase));
            int chip = s->code[i64_rem_euclid(idx, 1023)];
            int nav_pm = 1;
            if (s->nav == LPK_NAV_DUMMY) {
                nav_pm = orc_nav_bit_pm(s->nav_seed, f64_to_i64(floor(dt * NAV_BIT_RATE_HZ)));
            } else if (s->nav == LPK_NAV_FULL) {
                int64_t b = f64_to_i64(floor(dt * NAV_BIT_RATE_HZ));
                if (s->nav_n == 0) nav_pm = 1;
                else if (b < 0) nav_pm = s->nav_bits[0];
                else nav_pm = s->nav_bits[b < s->nav_n ? b : s->nav_n - 1];
            }
            re = (float)(chip * nav_pm);
            break;
        }
        }
        if (s->has_gate && !orc_gate_is_on(s, t)) { re = 0.0f; im = 0.0f; }
        out[2 * i] = re;
        out[2 * i + 1] = im;
    }
}

void orc_signal_free(orc_signal *s) {
    free(s->pm); free(s->bits); free(s->sym); free(s->nav_bits); free(s->gate_on);
    memset(s, 0, sizeof *s);
}

/* ======================= channel ======================= */
/* Antenna::amplitude_at, src/rx/mod.rs:48-58 */
float orc_antenna_amplitude(const orc_antenna *a, double elev_deg) {
    if (a->has_cutoff && elev_deg < a->cutoff_deg) return 0.0f;
    double dbi = (elev_deg >= 0.0) ? a->horizon_dbi + (a->peak_dbi - a->horizon_dbi) * (elev_deg / 90.0)
                                   : a->horizon_dbi - a->fb_db;
    return (float)pow(10.0, dbi / 20.0);
}

/* solve_emission_times_for, src/channel/mod.rs:49-101 */
void orc_solve_emission_times(const orc_traj *src, const double *obs, const double *t_rel_utc,
                              int64_t n, double epoch, int iterations,
                              double *t_emit, double *ranges) {
    double inv_c = 1.0 / SPEED_OF_LIGHT_M_S;
    for (int64_t i = 0; i < n; i++) {
        double tu = t_rel_utc[i];
        double ox = obs[i], oy = obs[n + i], oz = obs[2 * n + i];
        double t = tu - EMISSION_INITIAL_LAG_S;
        double r = 0.0;
        for (int it = 0; it < iterations; it++) {
            double p[3];
            orc_traj_position(src, epoch + t, p);
            double wtau = EARTH_ROTATION_RATE * (tu - t);
            double sx_rot = p[0] + wtau * p[1];
            double sy_rot = p[1] - wtau * p[0];
            double dx = sx_rot - ox;
            double dy = sy_rot - oy;
            double dz = p[2] - oz;
            r = sqrt(dx * dx + dy * dy + dz * dz);
            t = tu - r * inv_c;
        }
        t_emit[i] = t;
        ranges[i] = r;
    }
}

static void position_ld(const orc_traj *t, long double t_unix, long double out[3]) {
    if (t->kind != ORC_TRAJ_PRECOMPUTED) {
        double p[3];
        orc_traj_position(t, (double)t_unix, p);
        out[0] = p[0]; out[1] = p[1]; out[2] = p[2];
        return;
    }
    long double f = (t_unix - (long double)t->t0_unix) / (long double)t->dt_s;
    int64_t lo = (int64_t)floorl(f);
    if (lo < 0) lo = 0;
    if (lo > t->n - 2) lo = t->n - 2;
    long double frac = f - (long double)lo;
    if (frac < 0) frac = 0;
    if (frac > 1) frac = 1;
    for (int ax = 0; ax < 3; ax++) {
        const double *a = t->grid + ax * t->n;
        out[ax] = (long double)a[lo] * (1.0L - frac) + (long double)a[lo + 1] * frac;
    }
}

/* Converged light-time solve on the same trajectory model (lerp table,
 * linearised Sagnac), in 80-bit arithmetic: the FP64 delay truth. */
void orc_solve_converged(const orc_traj *src, const double *obs, const double *t_rel_utc,
                         int64_t n, double epoch, double tol_s, int max_iter,
                         double *t_emit, double *ranges, int32_t *iters_used) {
    for (int64_t i = 0; i < n; i++) {
        long double tu = t_rel_utc[i];
        long double ox = obs[i], oy = obs[n + i], oz = obs[2 * n + i];
        long double t = tu - (long double)EMISSION_INITIAL_LAG_S, r = 0;
        int it;
        for (it = 0; it < max_iter; it++) {
            long double p[3];
            position_ld(src, (long double)epoch + t, p);
            long double wtau = (long double)EARTH_ROTATION_RATE * (tu - t);
            long double dx = p[0] + wtau * p[1] - ox;
            long double dy = p[1] - wtau * p[0] - oy;
            long double dz = p[2] - oz;
            r = sqrtl(dx * dx + dy * dy + dz * dz);
            long double tn = tu - r / (long double)SPEED_OF_LIGHT_M_S;
            long double d = fabsl(tn - t);
            t = tn;
            if (d <= tol_s) { it++; break; }
        }
        t_emit[i] = (double)t;
        ranges[i] = (double)r;
        if (iters_used) iters_used[i] = it;
    }
}

/* accumulate_reporting_occlusion, src/channel/mod.rs:164-271 */
/* The mix loop of accumulate_reporting_occlusion, src/channel/mod.rs:236-268:
 * phase in f64, f64 sin/cos, f32 amplitude and complex MAC into acc. */
static void mix_into(float *acc, double src_carrier, const double *ranges, const float *bb, const float *gg,
                     const double *t_local, const double *delta_t, int64_t n, double lo_hz, double tx_power_w) {
    double wavelength_m = SPEED_OF_LIGHT_M_S / src_carrier;
    double tx_amplitude_v = sqrt(tx_power_w);
    double neg_tau_src = -TAU * src_carrier;
    double tau_if = TAU * (src_carrier - lo_hz);
    double amp_factor = (wavelength_m / (2.0 * TAU)) * tx_amplitude_v;
    double inv_c = 1.0 / SPEED_OF_LIGHT_M_S;
    for (int64_t i = 0; i < n; i++) {
        float g = gg ? gg[i] : 1.0f;
        if (g == 0.0f) continue;
        double r = ranges[i];
        double delay = r * inv_c;
        double phase = neg_tau_src * (delay + delta_t[i]) + tau_if * t_local[i];
        double sp = sin(phase), cp = cos(phase);
        float amplitude = (float)(amp_factor / r) * g;
        float br = bb[2 * i], bi = bb[2 * i + 1];
        float cpf = (float)cp, spf = (float)sp;
        acc[2 * i] = acc[2 * i] + amplitude * (br * cpf - bi * spf);
        acc[2 * i + 1] = acc[2 * i + 1] + amplitude * (br * spf + bi * cpf);
    }
}

int orc_accumulate(float *acc, const orc_signal *sig, const orc_traj *traj, const double *obs,
                   const double *t_local, const double *t_utc, const double *delta_t, int64_t n,
                   double lo_hz, double tx_power_w, double epoch, int iterations,
                   const orc_antenna *antenna) {
    double *t_emit = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
    double *ranges = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
    float *bb = (float *)malloc(sizeof(float) * 2 * (size_t)(n ? n : 1));
    float *gg = NULL;
    orc_solve_emission_times(traj, obs, t_utc, n, epoch, iterations, t_emit, ranges);
    orc_signal_eval(sig, t_emit, n, bb);
    int unoccluded = n > 0;
    if (antenna) {
        gg = (float *)malloc(sizeof(float) * (size_t)(n ? n : 1));
        double *abs_emit = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
        double *src = (double *)malloc(sizeof(double) * 3 * (size_t)(n ? n : 1));
        for (int64_t i = 0; i < n; i++) abs_emit[i] = epoch + t_emit[i];
        orc_traj_position_batch(traj, abs_emit, n, src);
        unoccluded = 0;
        for (int64_t i = 0; i < n; i++) {
            double ox = obs[i], oy = obs[n + i], oz = obs[2 * n + i];
            double on = sqrt(ox * ox + oy * oy + oz * oz);
            double dx = src[i] - ox, dy = src[n + i] - oy, dz = src[2 * n + i] - oz;
            double dn = sqrt(dx * dx + dy * dy + dz * dz);
            double sin_el = (dx * ox + dy * oy + dz * oz) / (dn * on);
            gg[i] = orc_antenna_amplitude(antenna, to_degrees(asin(f64_clamp(sin_el, -1.0, 1.0))));
            if (gg[i] != 0.0f) unoccluded = 1;
        }
        free(abs_emit);
        free(src);
    }
    mix_into(acc, sig->carrier_hz, ranges, bb, gg, t_local, delta_t, n, lo_hz, tx_power_w);
    free(t_emit); free(ranges); free(bb); free(gg);
    return unoccluded;
}

/* src/channel/mod.rs:310-312 */
double orc_thermal_noise_power_w(double temperature_k, double bandwidth_hz) {
    return BOLTZMANN * temperature_k * bandwidth_hz;
}

/* bands_overlap, src/pipeline.rs:70-75 */
int orc_bands_overlap(double tx_carrier, double tx_bw, double band_lo, double band_bw) {
    return fabs(tx_carrier - band_lo) <= 0.5 * (tx_bw + band_bw);
}

/* ======================= rx chain ======================= */
/* RxChain::from_config, src/rx/mod.rs:117-137 */
void orc_rx_chain_from_config(const lpk_frontend_cfg *fe, int has_frontend, orc_rx_chain *c) {
    memset(c, 0, sizeof *c);
    if (!has_frontend || !fe) return;
    if (fe->has_antenna) {
        c->has_antenna = 1;
        c->antenna.peak_dbi = fe->peak_dbi;
        c->antenna.horizon_dbi = fe->horizon_dbi;
        c->antenna.fb_db = fe->fb_db;
        c->antenna.has_cutoff = fe->has_cutoff;
        c->antenna.cutoff_deg = fe->cutoff_deg;
    }
    if (fe->has_gain) { c->post[c->n_post].kind = ORC_POST_GAIN; c->post[c->n_post++].a = fe->gain_db; }
    if (fe->has_nonlinearity) {
        c->post[c->n_post].kind = ORC_POST_NONLIN;
        c->post[c->n_post++].a = pow(10.0, (fe->iip3_dbm - 30.0) / 10.0);
    }
    if (fe->has_adc) {
        c->post[c->n_post].kind = ORC_POST_ADC;
        c->post[c->n_post].bits = fe->adc_bits;
        c->post[c->n_post++].a = fe->adc_full_scale_v;
    }
}

/* PostOp::apply, src/rx/mod.rs:83-101 */
void orc_rx_apply_post_sum(const orc_rx_chain *c, float *iq, int64_t n) {
    for (int k = 0; k < c->n_post; k++) {
        const orc_post_op *op = &c->post[k];
        if (op->kind == ORC_POST_GAIN) {
            float g = powf(10.0f, (float)(op->a / 20.0));
            for (int64_t i = 0; i < 2 * n; i++) iq[i] = iq[i] * g;
        } else if (op->kind == ORC_POST_NONLIN) {
            float kk = (float)(4.0 / 3.0 / op->a);
            for (int64_t i = 0; i < n; i++) {
                float re = iq[2 * i], im = iq[2 * i + 1];
                float f = 1.0f - kk * (re * re + im * im);
                iq[2 * i] = re * f;
                iq[2 * i + 1] = im * f;
            }
        } else {
            float fs = (float)op->a;
            uint32_t b = op->bits < 2 ? 2 : op->bits;
            float levels = (float)((1ULL << (b - 1)) - 1ULL);
            float lsb = fs / levels;
            for (int64_t i = 0; i < 2 * n; i++) iq[i] = roundf(f32_clamp(iq[i], -fs, fs) / lsb) * lsb;
        }
    }
}

int orc_adc_codes(const orc_rx_chain *c, const float *iq, int64_t n, int32_t *codes) {
    for (int k = c->n_post - 1; k >= 0; k--) {
        const orc_post_op *op = &c->post[k];
        if (op->kind != ORC_POST_ADC) continue;
        float fs = (float)op->a;
        uint32_t b = op->bits < 2 ? 2 : op->bits;
        float levels = (float)((1ULL << (b - 1)) - 1ULL);
        float lsb = fs / levels;
        for (int64_t i = 0; i < 2 * n; i++) codes[i] = (int32_t)roundf(iq[i] / lsb);
        return 1;
    }
    return 0;
}

/* ======================= clock ======================= */
#define FLICKER_RATE_HZ 128.0
#define FLICKER_POLES 20
#define FLICKER_F_LO 1e-4
#define FLICKER_BURN_STEPS 200000

typedef struct {
    double alpha[FLICKER_POLES], gain[FLICKER_POLES], state[FLICKER_POLES];
    double scale;
    orc_xoshiro rng;
    int64_t frontier;
    double delta_hi, delta_lo;
} orc_flicker;

struct orc_clock {
    double start_epoch, master_rate, initial_offset, y0, step_std;
    int has_walk;
    orc_xoshiro rng;
    int64_t frontier;
    double eps_hi, eps_lo;
    int has_flicker;
    orc_flicker flicker;
};

/* Flicker::poles / raw_step, src/clock/mod.rs:72-93 */
static void flicker_poles(double *alpha, double *gain) {
    double f_hi = FLICKER_RATE_HZ / 2.0;
    for (int j = 0; j < FLICKER_POLES; j++) {
        double f = FLICKER_F_LO * pow(f_hi / FLICKER_F_LO, (double)j / (double)(FLICKER_POLES - 1));
        double a = exp(-2.0 * M_PI * f / FLICKER_RATE_HZ);
        alpha[j] = a;
        gain[j] = sqrt(1.0 - a * a);
    }
}
static double flicker_raw_step(const double *alpha, const double *gain, double *state,
                               orc_xoshiro *rng) {
    double y = 0.0;
    for (int j = 0; j < FLICKER_POLES; j++) {
        state[j] = alpha[j] * state[j] + gain[j] * (0.0 + 1.0 * orc_std_normal(rng));
        y += state[j];
    }
    return y;
}
/* allan_dev_from_delta, src/clock/mod.rs:151-165 */
static double allan_dev_from_delta(const double *delta, int64_t len, int64_t m, double fc) {
    double tau = (double)m / fc;
    double sum = 0.0;
    int64_t cnt = 0;
    for (int64_t i = 0; i + 2 * m < len; i += m) {
        double d = delta[i + 2 * m] - 2.0 * delta[i + m] + delta[i];
        sum += d * d;
        cnt++;
    }
    return sqrt((sum / (double)(cnt > 1 ? cnt : 1)) / (2.0 * tau * tau));
}
/* Flicker::new, src/clock/mod.rs:95-128 */
static void flicker_init(orc_flicker *f, double floor_v, const orc_xoshiro *seed_rng) {
    flicker_poles(f->alpha, f->gain);
    orc_xoshiro crng = *seed_rng;
    orc_xoshiro_long_jump(&crng);
    double cstate[FLICKER_POLES] = {0};
    for (int i = 0; i < FLICKER_BURN_STEPS; i++) flicker_raw_step(f->alpha, f->gain, cstate, &crng);
    int64_t nc = 1 << 18;
    double *delta = (double *)calloc((size_t)nc, sizeof(double));
    double acc = 0.0;
    for (int64_t i = 1; i < nc; i++) {
        acc += flicker_raw_step(f->alpha, f->gain, cstate, &crng) / FLICKER_RATE_HZ;
        delta[i] = acc;
    }
    int64_t m = (int64_t)(2.0 * FLICKER_RATE_HZ);
    double measured = allan_dev_from_delta(delta, nc, m, FLICKER_RATE_HZ);
    if (measured < 1e-30) measured = 1e-30;
    free(delta);
    f->scale = floor_v / measured;
    f->rng = *seed_rng;
    orc_xoshiro_long_jump(&f->rng);
    orc_xoshiro_long_jump(&f->rng);
    memset(f->state, 0, sizeof f->state);
    for (int i = 0; i < FLICKER_BURN_STEPS; i++) flicker_raw_step(f->alpha, f->gain, f->state, &f->rng);
    f->frontier = -1;
    f->delta_hi = 0.0;
    f->delta_lo = 0.0;
}
/* Flicker::advance_to / delta_at, src/clock/mod.rs:130-148 */
static double flicker_delta_at(orc_flicker *f, double elapsed_s) {
    double x = (elapsed_s > 0.0 ? elapsed_s : 0.0) * FLICKER_RATE_HZ;
    int64_t m0 = f64_to_i64(floor(x));
    double frac = x - (double)m0;
    while (f->frontier < m0 + 1) {
        f->delta_lo = f->delta_hi;
        double y = flicker_raw_step(f->alpha, f->gain, f->state, &f->rng) * f->scale;
        f->delta_hi += y / FLICKER_RATE_HZ;
        f->frontier += 1;
    }
    return f->delta_lo * (1.0 - frac) + f->delta_hi * frac;
}

/* ClockStream::new, src/clock/mod.rs:268-295 */
orc_clock *orc_clock_new(const lpk_clock_cfg *spec, double start_epoch, double master_rate_hz,
                         uint64_t seed) {
    orc_clock *c = (orc_clock *)calloc(1, sizeof *c);
    c->start_epoch = start_epoch;
    c->master_rate = master_rate_hz;
    c->initial_offset = spec->initial_time_offset_s;
    c->y0 = spec->frequency_offset_y0;
    c->has_walk = spec->allan_deviation_1s > 0.0;
    c->step_std = c->has_walk ? spec->allan_deviation_1s / sqrt(master_rate_hz) : 0.0;
    orc_xoshiro_seed(&c->rng, seed);
    c->frontier = -1;
    if (spec->flicker_floor > 0.0) {
        c->has_flicker = 1;
        flicker_init(&c->flicker, spec->flicker_floor, &c->rng);
    }
    return c;
}
/* ClockStream::advance_to, src/clock/mod.rs:299-307 */
static void clock_advance_to(orc_clock *c, int64_t k) {
    /* without a walk every step keeps eps at 0: jump the frontier (exact) */
    if (!c->has_walk && c->frontier < k) {
        c->eps_lo = c->eps_hi;
        c->frontier = k;
        return;
    }
    while (c->frontier < k) {
        c->eps_lo = c->eps_hi;
        if (c->has_walk) c->eps_hi += 0.0 + c->step_std * orc_std_normal(&c->rng);
        c->frontier += 1;
    }
}
static double clock_det(const orc_clock *c, double e) { return c->initial_offset + c->y0 * e; }

/* ClockStream::delta_t_at_master_index, src/clock/mod.rs:317-324 */
double orc_clock_delta_t_at_master_index(orc_clock *c, int64_t k) {
    clock_advance_to(c, k > 0 ? k : 0);
    double eps = k < 0 ? 0.0 : c->eps_hi;
    double elapsed = (double)(k > 0 ? k : 0) / c->master_rate;
    double flick = c->has_flicker ? flicker_delta_at(&c->flicker, elapsed) : 0.0;
    return eps + flick + clock_det(c, elapsed);
}

/* ClockStream::delta_t_at, src/clock/mod.rs:326-346 */
double orc_clock_delta_t_at(orc_clock *c, double t) {
    double elapsed = t - c->start_epoch;
    double x = elapsed * c->master_rate;
    if (x <= 0.0) {
        clock_advance_to(c, 0);
        double flick = c->has_flicker ? flicker_delta_at(&c->flicker, 0.0) : 0.0;
        return c->eps_hi + flick + clock_det(c, 0.0);
    }
    int64_t k0 = f64_to_i64(floor(x));
    double frac = x - (double)k0;
    clock_advance_to(c, k0 + 1);
    double eps = c->eps_lo * (1.0 - frac) + c->eps_hi * frac;
    double flick = c->has_flicker ? flicker_delta_at(&c->flicker, elapsed) : 0.0;
    return eps + flick + clock_det(c, elapsed);
}
void orc_clock_free(orc_clock *c) { free(c); }

/* src/pipeline.rs:825-830 */
uint64_t orc_clock_seed(uint64_t base, uint64_t r_idx) { return base + 0xC10C000000000000ULL + r_idx; }
uint64_t orc_noise_seed(uint64_t base, uint64_t work_idx) { return base + work_idx; }

/* ======================= scene ======================= */
typedef struct {
    orc_signal sig;
    orc_traj traj;
    double power_w, bandwidth_hz;
} orc_tx;
typedef struct {
    orc_traj traj;
    lpk_clock_cfg clock;
    int n_bands;
    lpk_band_cfg *bands;
} orc_rx;
struct orc_scene {
    lpk_scene_cfg cfg;
    int n_tx, n_rx, n_work;
    orc_tx *tx;
    orc_rx *rx;
    int *work_r, *work_b;
};

/* SignalKind::default_bandwidth_hz, src/config/mod.rs:260-268 */
static double tx_bandwidth(const lpk_transmitter_cfg *t) {
    if (t->has_bandwidth) return t->bandwidth_hz;
    switch (t->kind) {
    case LPK_SIG_CW: return 0.0;
    case LPK_SIG_CA_CODE: return 2.0 * CA_CHIP_RATE_HZ;
    default: return 2.0 * t->rate_hz;
    }
}

void orc_scene_free(orc_scene *s) {
    if (!s) return;
    for (int i = 0; i < s->n_tx; i++) { orc_signal_free(&s->tx[i].sig); orc_traj_free(&s->tx[i].traj); }
    for (int i = 0; i < s->n_rx; i++) { orc_traj_free(&s->rx[i].traj); free(s->rx[i].bands); }
    free(s->tx); free(s->rx); free(s->work_r); free(s->work_b);
    free(s);
}

/* prepare, src/pipeline.rs:801-819 */
int orc_scene_prepare(const lpk_scene_cfg *cfg, orc_scene **out) {
    orc_scene *s = (orc_scene *)calloc(1, sizeof *s);
    s->cfg = *cfg;
    s->n_tx = cfg->n_transmitters;
    s->n_rx = cfg->n_receivers;
    s->tx = (orc_tx *)calloc((size_t)(s->n_tx ? s->n_tx : 1), sizeof(orc_tx));
    s->rx = (orc_rx *)calloc((size_t)(s->n_rx ? s->n_rx : 1), sizeof(orc_rx));
    int rc = 0;
    for (int i = 0; i < s->n_tx && !rc; i++) {
        const lpk_transmitter_cfg *t = &cfg->transmitters[i];
        rc = orc_traj_for_transmitter(&t->trajectory, cfg->epoch_unix, cfg->duration_s, &s->tx[i].traj);
        if (!rc) rc = orc_signal_build(t, cfg, &s->tx[i].sig);
        s->tx[i].power_w = pow(10.0, t->tx_power_dbw / 10.0);
        s->tx[i].bandwidth_hz = tx_bandwidth(t);
    }
    int nw = 0;
    for (int r = 0; r < s->n_rx && !rc; r++) {
        const lpk_receiver_cfg *rcfg = &cfg->receivers[r];
        if (rcfg->n_bands < 1) { rc = -1; break; }
        rc = orc_traj_for_receiver(&rcfg->trajectory, cfg->epoch_unix, &s->rx[r].traj);
        s->rx[r].clock = rcfg->clock;
        s->rx[r].n_bands = rcfg->n_bands;
        s->rx[r].bands = (lpk_band_cfg *)malloc(sizeof(lpk_band_cfg) * (size_t)rcfg->n_bands);
        memcpy(s->rx[r].bands, rcfg->bands, sizeof(lpk_band_cfg) * (size_t)rcfg->n_bands);
        nw += rcfg->n_bands;
    }
    if (rc) { orc_scene_free(s); return rc; }
    s->n_work = nw;
    s->work_r = (int *)malloc(sizeof(int) * (size_t)(nw ? nw : 1));
    s->work_b = (int *)malloc(sizeof(int) * (size_t)(nw ? nw : 1));
    int w = 0;
    for (int r = 0; r < s->n_rx; r++)
        for (int b = 0; b < s->rx[r].n_bands; b++) { s->work_r[w] = r; s->work_b[w] = b; w++; }
    *out = s;
    return 0;
}
int orc_scene_n_work(const orc_scene *s) { return s->n_work; }
int orc_scene_work(const orc_scene *s, int w, int *r, int *b) {
    if (w < 0 || w >= s->n_work) return -1;
    *r = s->work_r[w]; *b = s->work_b[w];
    return 0;
}
int64_t orc_band_n_samples(const orc_scene *s, int r, int b) {
    return (int64_t)llround(s->rx[r].bands[b].sample_rate_hz * s->cfg.duration_s);
}
static double band_bw(const lpk_band_cfg *b) { return b->has_bandwidth ? b->bandwidth_hz : b->sample_rate_hz; }
int orc_band_active(const orc_scene *s, int r, int b, int32_t *active, int cap) {
    const lpk_band_cfg *band = &s->rx[r].bands[b];
    int k = 0;
    for (int i = 0; i < s->n_tx; i++)
        if (orc_bands_overlap(s->tx[i].sig.carrier_hz, s->tx[i].bandwidth_hz, band->lo_carrier_hz,
                              band_bw(band))) {
            if (k < cap) active[k] = i;
            k++;
        }
    return k;
}
const orc_signal *orc_scene_signal(const orc_scene *s, int tx) { return &s->tx[tx].sig; }
const orc_traj *orc_scene_traj(const orc_scene *s, int tx) { return &s->tx[tx].traj; }
double orc_scene_tx_power_w(const orc_scene *s, int tx) { return s->tx[tx].power_w; }

typedef struct {
    const orc_scene *s;
    const int32_t *active;
    int na;
    float *contrib;
    int *unocc;
    const double *rxp, *t_local, *t_utc, *delta;
    int64_t clen;
    double lo, epoch;
    const orc_antenna *ant;
    int next;
    pthread_mutex_t mu;
} fan_job;

/* One worker of the per-transmitter fan-out: takes transmitters one at a
 * time (work stealing, as rayon does) into that transmitter's own buffer. */
static void *fan_worker(void *arg) {
    fan_job *j = (fan_job *)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int k = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (k >= j->na) break;
        const orc_tx *tx = &j->s->tx[j->active[k]];
        j->unocc[k] = orc_accumulate(j->contrib + (size_t)k * 2 * (size_t)j->clen, &tx->sig, &tx->traj,
                                     j->rxp, j->t_local, j->t_utc, j->delta, j->clen, j->lo,
                                     tx->power_w, j->epoch, NEWTON_ITERATIONS, j->ant);
    }
    return NULL;
}

/* generate_band, src/pipeline.rs:836-1019 (horizon gate off: it never
 * changes the samples). The per-transmitter fan-out runs on n_threads
 * pthreads (the reference's rayon par_iter, :944-959) into one buffer
 * per transmitter, reduced in fixed order (:966-977). sample_limit < 0
 * renders the whole band; otherwise only the first sample_limit samples. */
int orc_generate_band(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int work_idx,
                      int64_t chunk_samples, int n_threads, int noise_mode, int64_t sample_limit,
                      float *out, double *out_delta, uint8_t *unoccluded) {
    return orc_generate_band_window(s, r_idx, b_idx, seed_base, work_idx, chunk_samples, n_threads, noise_mode, 0,
                                    sample_limit, out, out_delta, unoccluded);
}

/* The same loop over band samples [sample_start, sample_start + sample_limit)
 * only (chunk boundaries at sample_start + k chunk_samples): the window a
 * render_window-style caller asks for (src/pipeline.rs:746-794). The
 * sequential AWGN stream cannot start mid-band, so a window that does not
 * start at 0 takes NOISE_NONE or NOISE_COUNTER only. */
int orc_generate_band_window(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int work_idx,
                             int64_t chunk_samples, int n_threads, int noise_mode, int64_t sample_start,
                             int64_t sample_limit, float *out, double *out_delta, uint8_t *unoccluded) {
    const orc_rx *rx = &s->rx[r_idx];
    const lpk_band_cfg *band = &rx->bands[b_idx];
    double epoch = s->cfg.epoch_unix;
    double fs = band->sample_rate_hz;
    int64_t n_band = orc_band_n_samples(s, r_idx, b_idx);
    if (sample_start < 0 || sample_start > n_band) return -2;
    if (sample_start > 0 && noise_mode == ORC_NOISE_SEQUENTIAL) return -3;
    int64_t n = n_band - sample_start;
    if (sample_limit >= 0 && sample_limit < n) n = sample_limit;
    double lo = band->lo_carrier_hz;
    double master = 0.0;
    for (int b = 0; b < rx->n_bands; b++) master = fmax(master, rx->bands[b].sample_rate_hz);
    orc_clock *clock = orc_clock_new(&rx->clock, 0.0, master, orc_clock_seed(seed_base, (uint64_t)r_idx));
    orc_xoshiro noise_rng;
    uint64_t nseed = orc_noise_seed(seed_base, (uint64_t)work_idx);
    orc_xoshiro_seed(&noise_rng, nseed);
    double noise_power = band->has_noise_power ? band->noise_power_w
                                               : orc_thermal_noise_power_w(band->noise_temperature_k, fs);
    int32_t active[256];
    int na = orc_band_active(s, r_idx, b_idx, active, 256);
    if (na > 256) { orc_clock_free(clock); return -1; }
    orc_rx_chain chain;
    orc_rx_chain_from_config(&band->frontend, band->has_frontend, &chain);
    if (unoccluded) memset(unoccluded, 0, (size_t)(na ? na : 1));
    if (chunk_samples < 1) chunk_samples = 1;
    int64_t cap = chunk_samples < n ? chunk_samples : (n > 0 ? n : 1);
    double *t_local = (double *)malloc(sizeof(double) * (size_t)cap);
    double *delta = (double *)malloc(sizeof(double) * (size_t)cap);
    double *t_utc = (double *)malloc(sizeof(double) * (size_t)cap);
    double *t_abs = (double *)malloc(sizeof(double) * (size_t)cap);
    double *rxp = (double *)malloc(sizeof(double) * 3 * (size_t)cap);
    float *contrib = (float *)malloc(sizeof(float) * 2 * (size_t)cap * (size_t)(na ? na : 1));
    int *unocc_chunk = (int *)malloc(sizeof(int) * (size_t)(na ? na : 1));
    float noise_std = (float)sqrt(noise_power / 2.0);
    for (int64_t i0 = 0; i0 < n; i0 += chunk_samples) {
        int64_t i1 = i0 + chunk_samples < n ? i0 + chunk_samples : n;
        int64_t clen = i1 - i0;
        for (int64_t j = 0; j < clen; j++) t_local[j] = (double)(sample_start + i0 + j) / fs;
        for (int64_t j = 0; j < clen; j++) delta[j] = orc_clock_delta_t_at(clock, t_local[j]);
        for (int64_t j = 0; j < clen; j++) t_utc[j] = t_local[j] - delta[j];
        for (int64_t j = 0; j < clen; j++) t_abs[j] = epoch + t_utc[j];
        orc_traj_position_batch(&rx->traj, t_abs, clen, rxp);
        memset(contrib, 0, sizeof(float) * 2 * (size_t)clen * (size_t)(na ? na : 1));
        fan_job job = {s, active, na, contrib, unocc_chunk, rxp, t_local, t_utc, delta, clen, lo,
                       epoch, chain.has_antenna ? &chain.antenna : NULL, 0, PTHREAD_MUTEX_INITIALIZER};
        int nt = n_threads > 1 ? (n_threads < na ? n_threads : na) : 1;
        if (nt <= 1) {
            fan_worker(&job);
        } else {
            pthread_t th[64];
            if (nt > 64) nt = 64;
            for (int t = 0; t < nt; t++) pthread_create(&th[t], NULL, fan_worker, &job);
            for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
        }
        float *acc = out + 2 * i0;
        for (int64_t j = 0; j < 2 * clen; j++) acc[j] = 0.0f;
        for (int k = 0; k < na; k++) {
            const float *c = contrib + (size_t)k * 2 * (size_t)clen;
            for (int64_t j = 0; j < 2 * clen; j++) acc[j] = acc[j] + c[j];
            if (unoccluded) unoccluded[k] |= (uint8_t)unocc_chunk[k];
        }
        if (noise_mode == ORC_NOISE_SEQUENTIAL) { /* add_awgn_at_power, channel/mod.rs:323-334 */
            for (int64_t j = 0; j < clen; j++) {
                acc[2 * j] += 0.0f + noise_std * (float)orc_std_normal(&noise_rng);
                acc[2 * j + 1] += 0.0f + noise_std * (float)orc_std_normal(&noise_rng);
            }
        } else if (noise_mode == ORC_NOISE_COUNTER && noise_power > 0.0) {
            for (int64_t j = 0; j < clen; j++) {
                float zr, zi;
                orc_noise_pair(nseed, sample_start + i0 + j, &zr, &zi);
                acc[2 * j] += noise_std * zr;
                acc[2 * j + 1] += noise_std * zi;
            }
        }
        orc_rx_apply_post_sum(&chain, acc, clen);
        if (out_delta) memcpy(out_delta + i0, delta, sizeof(double) * (size_t)clen);
    }
    free(t_local); free(delta); free(t_utc); free(t_abs); free(rxp); free(contrib); free(unocc_chunk);
    orc_clock_free(clock);
    return 0;
}

/* Single-thread cost of the sections of generate_band's loop
 * (src/pipeline.rs:911-983) on the first n samples of band (r_idx, b_idx),
 * in one chunk, with the horizon gate off and no antenna: ns_out[0] clock
 * offsets (per band sample), [1] receiver positions (per band sample),
 * [2] emission solves, [3] baseband, [4] mix (phase, f64 sin/cos, f32 MAC)
 * (each per tx-rx sample), [5] fixed-order sum (per band sample), [6] AWGN
 * (per band sample), [7] the largest |carrier phase| argument handed to
 * sin/cos (rad). Test infrastructure: times the restatement, not the
 * reference binary. */
static double now_ns(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return 1e9 * (double)ts.tv_sec + (double)ts.tv_nsec;
}
int orc_profile_sections(const orc_scene *s, int r_idx, int b_idx, uint64_t seed_base, int64_t n, double *ns_out) {
    const orc_rx *rx = &s->rx[r_idx];
    const lpk_band_cfg *band = &rx->bands[b_idx];
    int64_t nb = orc_band_n_samples(s, r_idx, b_idx);
    if (n > nb) n = nb;
    if (n <= 0) return -1;
    double fs = band->sample_rate_hz, epoch = s->cfg.epoch_unix, lo = band->lo_carrier_hz;
    double master = 0.0;
    for (int b = 0; b < rx->n_bands; b++) master = fmax(master, rx->bands[b].sample_rate_hz);
    int32_t active[256];
    int na = orc_band_active(s, r_idx, b_idx, active, 256);
    if (na > 256) return -1;
    double *t_local = malloc(sizeof(double) * (size_t)n), *delta = malloc(sizeof(double) * (size_t)n);
    double *t_utc = malloc(sizeof(double) * (size_t)n), *t_abs = malloc(sizeof(double) * (size_t)n);
    double *rxp = malloc(sizeof(double) * 3 * (size_t)n), *te = malloc(sizeof(double) * (size_t)n);
    double *rg = malloc(sizeof(double) * (size_t)n);
    float *bb = malloc(sizeof(float) * 2 * (size_t)n);
    float *contrib = calloc(2 * (size_t)n * (size_t)(na ? na : 1), sizeof(float));
    float *acc = malloc(sizeof(float) * 2 * (size_t)n);
    for (int i = 0; i < 8; i++) ns_out[i] = 0.0;
    double t0 = now_ns();
    orc_clock *clock = orc_clock_new(&rx->clock, 0.0, master, orc_clock_seed(seed_base, (uint64_t)r_idx));
    for (int64_t j = 0; j < n; j++) t_local[j] = (double)j / fs;
    for (int64_t j = 0; j < n; j++) delta[j] = orc_clock_delta_t_at(clock, t_local[j]);
    double t1 = now_ns();
    for (int64_t j = 0; j < n; j++) t_utc[j] = t_local[j] - delta[j];
    for (int64_t j = 0; j < n; j++) t_abs[j] = epoch + t_utc[j];
    orc_traj_position_batch(&rx->traj, t_abs, n, rxp);
    double t2 = now_ns();
    ns_out[0] = (t1 - t0) / (double)n;
    ns_out[1] = (t2 - t1) / (double)n;
    double solve = 0.0, base = 0.0, mix = 0.0, big = 0.0;
    for (int k = 0; k < na; k++) {
        const orc_tx *tx = &s->tx[active[k]];
        double a = now_ns();
        orc_solve_emission_times(&tx->traj, rxp, t_utc, n, epoch, NEWTON_ITERATIONS, te, rg);
        double b = now_ns();
        orc_signal_eval(&tx->sig, te, n, bb);
        double c = now_ns();
        mix_into(contrib + (size_t)k * 2 * (size_t)n, tx->sig.carrier_hz, rg, bb, NULL, t_local, delta, n, lo,
                 tx->power_w);
        double d = now_ns();
        solve += b - a;
        base += c - b;
        mix += d - c;
        double nts = -TAU * tx->sig.carrier_hz, tif = TAU * (tx->sig.carrier_hz - lo);
        for (int64_t j = 0; j < n; j += 997) big = fmax(big, fabs(nts * (rg[j] / SPEED_OF_LIGHT_M_S + delta[j]) +
                                                              tif * t_local[j]));
    }
    double t3 = now_ns();
    for (int64_t j = 0; j < 2 * n; j++) acc[j] = 0.0f;
    for (int k = 0; k < na; k++) {
        const float *c = contrib + (size_t)k * 2 * (size_t)n;
        for (int64_t j = 0; j < 2 * n; j++) acc[j] = acc[j] + c[j];
    }
    double t4 = now_ns();
    orc_xoshiro noise_rng;
    orc_xoshiro_seed(&noise_rng, 12345);
    for (int64_t j = 0; j < n; j++) {
        acc[2 * j] += 0.0f + 1e-7f * (float)orc_std_normal(&noise_rng);
        acc[2 * j + 1] += 0.0f + 1e-7f * (float)orc_std_normal(&noise_rng);
    }
    double t5 = now_ns();
    double ntx = (double)n * (double)(na ? na : 1);
    ns_out[2] = solve / ntx;
    ns_out[3] = base / ntx;
    ns_out[4] = mix / ntx;
    ns_out[5] = (t4 - t3) / (double)n;
    ns_out[6] = (t5 - t4) / (double)n;
    ns_out[7] = big;
    orc_clock_free(clock);
    free(t_local); free(delta); free(t_utc); free(t_abs); free(rxp); free(te); free(rg); free(bb); free(contrib);
    free(acc);
    return 0;
}
