// lpk_device.cuh — device-side data layout and per-sample arithmetic of the
// lipika fan-out, for sm_100a.
//
// The "reference" functions below perform every f64/f32 operation of the
// reference's per-sample code in the reference's order with explicit
// round-to-nearest intrinsics (__dadd_rn, __dmul_rn, ...), so the compiler
// never fuses them into FMAs: emission times, ranges and every table index
// are bit-identical to the CPU path. Only sin/cos/asin/pow come from CUDA's
// math library instead of glibc (last-ulp differences, well inside the
// 1e-5 IQ tolerance).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lpk {

constexpr double kTau = 6.283185307179586476925286766559;
constexpr double kSpeedOfLight = 299792458.0;          // src/lib.rs:53
constexpr double kEmissionLag = 0.07;                  // src/channel/mod.rs:23
constexpr double kEarthRate = 7.2921151467e-5;         // src/channel/mod.rs:27
constexpr double kCaChipRate = 1023000.0;              // src/signal/ca_code.rs:23
constexpr double kNavBitRate = 50.0;                   // src/signal/ca_code.rs:27
constexpr double kFlickerRate = 128.0;                 // src/clock/mod.rs:67 (flicker track rate)

enum SigKind : int32_t { kCw = 0, kBpsk = 1, kOok = 2, kQam16 = 3, kCa = 4 };
enum NavKind : int32_t { kNavOff = 0, kNavDummy = 1, kNavFull = 2 };

// One transmitter in device memory. Tables live in the context's scene
// arena; the trajectory grid is interleaved (x, y, z, pad) per point so a
// lerp reads one 64-byte line for the two bracketing points.
// 16-byte aligned so that anything staged after an array of DevTx in
// shared memory (the 16-byte aligned anchor records) stays aligned.
struct __align__(16) DevTx {
    int32_t traj_kind, sig_kind, nav_kind, has_repeat;
    int32_t has_gate, gate_n, cw_anchored, reserved;
    double sx, sy, sz;                  // stationary ECEF
    double t0, dt, inv_dt;              // grid start, step, 1/step (batch query)
    int64_t grid_n;
    const double4 *grid;                // grid_n points
    double carrier, neg_tau_src, amp_factor;
    double epoch_rel, rate;
    int64_t repeat_from, n_sym;
    const int8_t *pm;                   // bpsk ±1
    const uint8_t *ook;                 // ook 0/1
    const float2 *sym;                  // qam16
    uint32_t chip_neg[32];              // ca: bit i set <=> chip i == -1
    uint64_t nav_seed;
    const int8_t *nav_bits;
    int64_t nav_n;
    double cw_omega, cw_phase0;
    double gate_period, gate_phase;
    const double2 *gate_on;             // (start, end)
    double max_speed, max_radius;       // bounds of the trajectory table (horizon gate): longest
                                        // segment / dt and largest |P| (NaN if not finite)
};
static_assert(sizeof(DevTx) % 16 == 0, "DevTx arrays must keep 16-byte alignment");

// A circular Keplerian orbit (CircularKeplerian, src/geometry/kepler.rs:32-85)
// with its per-orbit constants computed once on the host: radius, mean
// motion, true anomaly at epoch (rad), sines and cosines of inclination and
// RAAN, epoch (unix s).
struct DevOrbit {
    double r, mm, nu0, si, ci, so, co, epoch;
};

// CircularKeplerian::position_ecef at orbit time e = t - epoch, in the
// host's operation order (explicit rounding); with vel, also the ECEF
// velocity, the exact time derivative of that expression (ν' = mean motion,
// θ' = ω⊕).
__device__ __forceinline__ void kepler_at(const DevOrbit &k, double e, double &x, double &y, double &z,
                                          double *vel = nullptr) {
    const double nu = __dadd_rn(k.nu0, __dmul_rn(k.mm, e));
    double snu, cnu;
    sincos(nu, &snu, &cnu);
    const double xp = __dmul_rn(k.r, cnu), yp = __dmul_rn(k.r, snu);
    const double y1 = __dmul_rn(yp, k.ci), z1 = __dmul_rn(yp, k.si);
    const double xe = __dsub_rn(__dmul_rn(xp, k.co), __dmul_rn(y1, k.so));
    const double ye = __dadd_rn(__dmul_rn(xp, k.so), __dmul_rn(y1, k.co));
    const double th = __dmul_rn(kEarthRate, e);
    double s, c;
    sincos(th, &s, &c);
    x = __dadd_rn(__dmul_rn(xe, c), __dmul_rn(ye, s));
    y = __dadd_rn(__dmul_rn(-xe, s), __dmul_rn(ye, c));
    z = z1;
    if (vel) {
        const double xpd = -yp * k.mm, ypd = xp * k.mm;
        const double y1d = ypd * k.ci;
        const double xed = xpd * k.co - y1d * k.so, yed = xpd * k.so + y1d * k.co;
        vel[0] = xed * c + yed * s + y * kEarthRate;
        vel[1] = -xed * s + yed * c - x * kEarthRate;
        vel[2] = ypd * k.si;
    }
}

// Per-band constants (host-computed where the reference computes them once).
struct DevBand {
    double epoch, fs, lo, inv_c;
    int64_t i0, n;
    int32_t rx_kind, clock_mode;
    double rx[3];
    double clock_offset, clock_y0;
    const double *delta;                // n (clock mode HOST)
    const double *rxpos;                // (3, n) (rx PER_SAMPLE)
    const double *eps;                  // walk ε on master indices [eps_k0, ...) (DEVICE_WALK)
    const double *eps_carry;            // non-NULL: eps holds the in-block prefix P_b(k) and
                                        // ε(k) = eps_carry[b] ⊕ P_b(k), b the scan block of k
    int64_t eps_k0;
    double fm;                          // master (walk) rate
    const double *flicker;              // coarse flicker track points [flicker_m0, flicker_m0 + flicker_n)
                                        // (DETERMINISTIC / DEVICE_WALK; NULL: no flicker)
    int64_t flicker_m0, flicker_n;
    float noise_std;                    // sqrt(P/2) as f32; 0 = no noise
    int32_t has_noise;
    uint64_t noise_seed;
    int32_t has_antenna, has_cutoff;
    double ant_peak, ant_horizon, ant_fb, ant_cutoff;
    int32_t n_post, reserved;
    unsigned long long *gate_stats;     // horizon gate counters (tested, skipped) or NULL
    uint32_t *unocc_words;              // split kernel: per active transmitter, set when any sample
                                        // has a non-zero antenna gain (NULL: not reported)
    unsigned long long *acc_stats;      // split kernel in accuracy mode: (max delay error, max phase
                                        // error) as double bits, (fast-path, exact-path) sample counts
    int32_t post_kind[3];
    float post_a[3], post_b[3];         // gain: g | nonlin: k | adc: fs, lsb
    DevOrbit rx_orb;                    // rx kind KEPLER: the receiver's orbit
    double rx_de;                       // KEPLER: epoch - rx_orb.epoch (exact), so the orbit time of
                                        // epoch-relative UTC tu is rx_de + tu without rounding epoch + tu
    int32_t rx_split_ok;                // KEPLER: fl(fl(epoch + tu) - orbit epoch) is exact for every tu of
                                        // the scene, so the split path's smooth receiver model holds
    int32_t rx_reserved;
};
static_assert(sizeof(DevBand) % 8 == 0, "DevBand is staged in 8-byte words");

// ---------------------------------------------------------------- helpers
// Read-only load of one 32-byte grid point as two 16-byte loads.
__device__ __forceinline__ double4 load_point(const double4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ double f64_rem_euclid(double a, double b) {
    double r = fmod(a, b);
    return (r < 0.0) ? __dadd_rn(r, fabs(b)) : r;
}
__device__ __forceinline__ int64_t i64_rem_euclid(int64_t a, int64_t b) {
    int64_t r = a % b;
    if (r < 0) r = (b < 0) ? r - b : r + b;
    return r;
}
// Rust `f64 as i64` (saturating, NaN -> 0) == PTX cvt.rzi.s64.f64.
__device__ __forceinline__ int64_t floor_to_i64(double x) { return __double2ll_rz(floor(x)); }

// PrecomputedTrajectory::position_ecef (src/geometry/precomputed.rs:111-121).
__device__ __forceinline__ void traj_position(const DevTx &tx, double t_unix, double &x, double &y,
                                              double &z) {
    if (tx.traj_kind == 0) { x = tx.sx; y = tx.sy; z = tx.sz; return; }
    double f = __ddiv_rn(__dsub_rn(t_unix, tx.t0), tx.dt);
    int64_t lo = floor_to_i64(f);
    lo = lo < 0 ? 0 : lo;
    lo = lo > tx.grid_n - 2 ? tx.grid_n - 2 : lo;
    double frac = __dsub_rn(f, (double)lo);
    frac = frac < 0.0 ? 0.0 : frac;
    frac = frac > 1.0 ? 1.0 : frac;
    double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
    double omf = __dsub_rn(1.0, frac);
    x = __dadd_rn(__dmul_rn(a.x, omf), __dmul_rn(b.x, frac));
    y = __dadd_rn(__dmul_rn(a.y, omf), __dmul_rn(b.y, frac));
    z = __dadd_rn(__dmul_rn(a.z, omf), __dmul_rn(b.z, frac));
}

// position_ecef_batch of the same table (precomputed.rs:136-153): scales by
// the precomputed 1/dt instead of dividing.
__device__ __forceinline__ void traj_position_batch(const DevTx &tx, double t_unix, double &x,
                                                    double &y, double &z) {
    if (tx.traj_kind == 0) { x = tx.sx; y = tx.sy; z = tx.sz; return; }
    double f = __dmul_rn(__dsub_rn(t_unix, tx.t0), tx.inv_dt);
    int64_t lo = floor_to_i64(f);
    lo = lo < 0 ? 0 : lo;
    lo = lo > tx.grid_n - 2 ? tx.grid_n - 2 : lo;
    double frac = __dsub_rn(f, (double)lo);
    frac = frac < 0.0 ? 0.0 : frac;
    frac = frac > 1.0 ? 1.0 : frac;
    double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
    double omf = __dsub_rn(1.0, frac);
    x = __dadd_rn(__dmul_rn(a.x, omf), __dmul_rn(b.x, frac));
    y = __dadd_rn(__dmul_rn(a.y, omf), __dmul_rn(b.y, frac));
    z = __dadd_rn(__dmul_rn(a.z, omf), __dmul_rn(b.z, frac));
}

// solve_emission_times_for (src/channel/mod.rs:70-99): fixed-point
// iterations from t_utc - 70 ms with the linearised Sagnac rotation.
__device__ __forceinline__ void solve_reference(const DevTx &tx, double tu, double ox, double oy,
                                                double oz, double epoch, int iterations,
                                                double inv_c, double &t_emit, double &range) {
    double t = __dsub_rn(tu, kEmissionLag);
    double r = 0.0;
    for (int it = 0; it < iterations; ++it) {
        double sx, sy, sz;
        traj_position(tx, __dadd_rn(epoch, t), sx, sy, sz);
        double wtau = __dmul_rn(kEarthRate, __dsub_rn(tu, t));
        double sxr = __dadd_rn(sx, __dmul_rn(wtau, sy));
        double syr = __dsub_rn(sy, __dmul_rn(wtau, sx));
        double dx = __dsub_rn(sxr, ox), dy = __dsub_rn(syr, oy), dz = __dsub_rn(sz, oz);
        r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        t = __dsub_rn(tu, __dmul_rn(r, inv_c));
    }
    t_emit = t;
    range = r;
}

// NavData::bit_pm (src/signal/ca_code.rs:94-108).
__device__ __forceinline__ int nav_bit_pm(uint64_t seed, int64_t bit_idx) {
    int64_t pos = i64_rem_euclid(bit_idx, 300);
    uint32_t bit;
    if (pos < 8) {
        bit = (0xD1u >> pos) & 1u;  // preamble 1,0,0,0,1,0,1,1 read LSB-first
    } else {
        uint64_t x = seed ^ ((uint64_t)bit_idx * 0x9E3779B97F4A7C15ULL);
        x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ULL;
        x ^= x >> 27; x *= 0x94D049BB133111EBULL;
        x ^= x >> 31;
        bit = (uint32_t)(x & 1);
    }
    return 1 - 2 * (int)bit;
}

// BurstGate::is_on (src/signal/gate.rs:71-77).
__device__ __forceinline__ bool gate_is_on(const DevTx &tx, double t) {
    double u = f64_rem_euclid(__dadd_rn(t, tx.gate_phase), tx.gate_period);
    if (u >= tx.gate_period) u = 0.0;
    for (int i = 0; i < tx.gate_n; ++i) {
        double2 on = tx.gate_on[i];
        if (u >= on.x && u < on.y) return true;
    }
    return false;
}

// The chip (±1) of a C/A code at raw chip count idx (ca_code.rs:170-174).
__device__ __forceinline__ int ca_chip(const DevTx &tx, int64_t idx) {
    int64_t m = (idx >= 0) ? (idx % 1023) : i64_rem_euclid(idx, 1023);
    uint32_t w = tx.chip_neg[m >> 5];
    return ((w >> (m & 31)) & 1u) ? -1 : 1;
}

// evaluate_baseband_batch for one emission time: cw.rs:41-52, bpsk.rs:58-71,
// ook.rs:60-74, qam16.rs:96-109, ca_code.rs:167-193, gate.rs:91-105.
__device__ __forceinline__ float2 baseband(const DevTx &tx, double t) {
    float re = 0.0f, im = 0.0f;
    switch (tx.sig_kind) {
    case kCw: {
        float ph = tx.cw_anchored
                       ? (float)f64_rem_euclid(__dadd_rn(__dmul_rn(tx.cw_omega, t), tx.cw_phase0), kTau)
                       : (float)__dmul_rn(tx.cw_omega, t);
        float s, c;
        sincosf(ph, &s, &c);
        re = c;
        im = s;
        break;
    }
    case kBpsk:
    case kOok:
    case kQam16: {
        int64_t raw = floor_to_i64(__dmul_rn(__dsub_rn(t, tx.epoch_rel), tx.rate));
        int64_t k = -1;
        if (!tx.has_repeat) {
            if (raw >= 0 && raw < tx.n_sym) k = raw;
        } else if (tx.n_sym > 0) {
            k = i64_rem_euclid((int64_t)((uint64_t)raw + (uint64_t)tx.repeat_from), tx.n_sym);
        }
        if (k >= 0) {
            if (tx.sig_kind == kBpsk) re = (float)__ldg(tx.pm + k);
            else if (tx.sig_kind == kOok) re = (float)__ldg(tx.ook + k);
            else { float2 s = __ldg(tx.sym + k); re = s.x; im = s.y; }
        }
        break;
    }
    case kCa: {
        double dt = __dsub_rn(t, tx.epoch_rel);
        int chip = ca_chip(tx, floor_to_i64(__dmul_rn(dt, kCaChipRate)));
        int nav = 1;
        if (tx.nav_kind == kNavDummy) {
            nav = nav_bit_pm(tx.nav_seed, floor_to_i64(__dmul_rn(dt, kNavBitRate)));
        } else if (tx.nav_kind == kNavFull) {
            int64_t b = floor_to_i64(__dmul_rn(dt, kNavBitRate));
            if (tx.nav_n == 0) nav = 1;
            else if (b < 0) nav = tx.nav_bits[0];
            else nav = tx.nav_bits[b < tx.nav_n ? b : tx.nav_n - 1];
        }
        re = (float)(chip * nav);
        break;
    }
    default:
        break;
    }
    if (tx.has_gate && !gate_is_on(tx, t)) { re = 0.0f; im = 0.0f; }
    return make_float2(re, im);
}

// Antenna::amplitude_at after the elevation geometry of
// accumulate_reporting_occlusion (channel/mod.rs:190-203, rx/mod.rs:48-58).
// Arrival elevation (degrees) of the source at absolute emission time
// t_emit_abs seen from O, against the geocentric up O/|O|.
__device__ __forceinline__ double antenna_elevation(const DevTx &tx, double t_emit_abs, double ox, double oy,
                                                   double oz) {
    double sx, sy, sz;
    traj_position_batch(tx, t_emit_abs, sx, sy, sz);
    double on = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(ox, ox), __dmul_rn(oy, oy)), __dmul_rn(oz, oz)));
    double dx = __dsub_rn(sx, ox), dy = __dsub_rn(sy, oy), dz = __dsub_rn(sz, oz);
    double dn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    double se = __ddiv_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, ox), __dmul_rn(dy, oy)), __dmul_rn(dz, oz)),
                          __dmul_rn(dn, on));
    se = se < -1.0 ? -1.0 : (se > 1.0 ? 1.0 : se);
    return __dmul_rn(asin(se), 57.2957795130823208767981548141051703);
}

// Antenna::amplitude_at (src/rx/mod.rs:48-58) at elevation el (degrees).
__device__ __forceinline__ float antenna_pattern(const DevBand &b, double el) {
    if (b.has_cutoff && el < b.ant_cutoff) return 0.0f;
    double dbi = (el >= 0.0)
                     ? __dadd_rn(b.ant_horizon, __dmul_rn(__dsub_rn(b.ant_peak, b.ant_horizon), __ddiv_rn(el, 90.0)))
                     : __dsub_rn(b.ant_horizon, b.ant_fb);
    return (float)pow(10.0, __ddiv_rn(dbi, 20.0));
}

__device__ __forceinline__ float antenna_gain(const DevTx &tx, const DevBand &b, double t_emit_abs,
                                              double ox, double oy, double oz) {
    return antenna_pattern(b, antenna_elevation(tx, t_emit_abs, ox, oy, oz));
}

// ---------------------------------------------------------------- noise
// Philox4x32-10 (Salmon et al., SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        if (round > 0) { k.x += 0x9E3779B9u; k.y += 0xBB67AE85u; }
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// t_local = i / fs (src/pipeline.rs:918), correctly rounded, without a
// division instruction sequence: with y = RN(1/fs), q = RN(i y) is within
// an ulp of i / fs, the remainder r = i - q fs is exact in one fma, and
// RN(q + r y) is the correctly rounded quotient (Markstein, IBM J. Res. Dev.
// 34, 1990). y comes from __drcp_rn, once per tile.
__device__ __forceinline__ double sample_time(double i, double fs, double rfs) {
    const double q = __dmul_rn(i, rfs);
    const double r = __fma_rn(-q, fs, i);
    return __fma_rn(r, rfs, q);
}

// AWGN for (seed, global band-sample index): one Philox block per pair of
// indices 2p, 2p+1 (words 0-1 for 2p, words 2-3 for 2p+1), Box–Muller in
// f32. Counter-based, so chunking cannot change it.
__device__ __forceinline__ float2 box_muller(uint32_t a, uint32_t b) {
    float u1 = __fmul_rn(__fadd_rn((float)(a >> 8), 1.0f), 0x1.0p-24f);
    float u2 = __fmul_rn((float)(b >> 8), 0x1.0p-24f);
    float rr = sqrtf(__fmul_rn(-2.0f, logf(u1)));
    // angle uniform on [-pi, pi), where the hardware sin/cos approximation
    // holds its 2^-21.4 absolute error bound
    float ang = __fsub_rn(__fmul_rn(6.28318548f, u2), 3.14159274f);
    float s, c;
    __sincosf(ang, &s, &c);
    return make_float2(__fmul_rn(rr, c), __fmul_rn(rr, s));
}
__device__ __forceinline__ uint4 noise_block(uint64_t seed, int64_t g) {
    const uint64_t p = (uint64_t)g >> 1;
    return philox4x32_10(make_uint4((uint32_t)p, (uint32_t)(p >> 32), 0x4E4F4953u, 0u),
                         make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}
__device__ __forceinline__ float2 noise_pair(uint64_t seed, int64_t g) {
    const uint4 x = noise_block(seed, g);
    return (g & 1) ? box_muller(x.z, x.w) : box_muller(x.x, x.y);
}

// Increments σ·z_k of the receiver clock's white-FM walk at master indices
// k = 4q .. 4q+3: one Philox block (counter q, tag "CLOK", keyed by the
// clock seed) gives two Box–Muller pairs in f32, with the angle uniform on
// [-π, π) and the hardware approximations of log, sin and cos (absolute
// error ~2^-21, far below what the walk's moments resolve). Counter-based,
// so any chunking or GPU regenerates the same walk.
__device__ __forceinline__ void walk_increments4(uint64_t seed, int64_t q, double sigma, double z[4]) {
    const uint4 x = philox4x32_10(make_uint4((uint32_t)(uint64_t)q, (uint32_t)((uint64_t)q >> 32), 0x434C4F4Bu, 0u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const uint32_t ua[2] = {x.x, x.z}, ub[2] = {x.y, x.w};
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const float u1 = __fmul_rn(__fadd_rn((float)(ua[p] >> 8), 1.0f), 0x1.0p-24f);
        const float u2 = __fmul_rn((float)(ub[p] >> 8), 0x1.0p-24f);
        const float r = sqrtf(__fmul_rn(-2.0f, __logf(u1)));
        float sn, cs;
        __sincosf(__fadd_rn(__fmul_rn(6.28318548f, u2), -3.14159274f), &sn, &cs);
        z[2 * p] = __dmul_rn(sigma, (double)__fmul_rn(r, cs));
        z[2 * p + 1] = __dmul_rn(sigma, (double)__fmul_rn(r, sn));
    }
}

// PostOp::apply in chain order (rx/mod.rs:83-101), on one band sample.
__device__ __forceinline__ float2 band_post(const DevBand &b, float re, float im);

// AWGN then the receiver chain (channel/mod.rs:323-334, rx/mod.rs:83-101),
// on one band sample.
__device__ __forceinline__ float2 band_epilogue(const DevBand &b, float re, float im, int64_t g) {
    if (b.has_noise) {
        float2 z = noise_pair(b.noise_seed, g);
        re = __fadd_rn(re, __fmul_rn(b.noise_std, z.x));
        im = __fadd_rn(im, __fmul_rn(b.noise_std, z.y));
    }
    return band_post(b, re, im);
}

// The same on the band-sample pair (g, g+1), g even: one Philox block.
__device__ __forceinline__ void band_epilogue2(const DevBand &b, float re0, float im0, float re1, float im1,
                                               int64_t g, float2 &o0, float2 &o1) {
    if (b.has_noise) {
        const uint4 x = noise_block(b.noise_seed, g);
        const float2 z0 = box_muller(x.x, x.y), z1 = box_muller(x.z, x.w);
        re0 = __fadd_rn(re0, __fmul_rn(b.noise_std, z0.x));
        im0 = __fadd_rn(im0, __fmul_rn(b.noise_std, z0.y));
        re1 = __fadd_rn(re1, __fmul_rn(b.noise_std, z1.x));
        im1 = __fadd_rn(im1, __fmul_rn(b.noise_std, z1.y));
    }
    o0 = band_post(b, re0, im0);
    o1 = band_post(b, re1, im1);
}

__device__ __forceinline__ float2 band_post(const DevBand &b, float re, float im) {
    for (int k = 0; k < b.n_post; ++k) {
        if (b.post_kind[k] == 0) {
            re = __fmul_rn(re, b.post_a[k]);
            im = __fmul_rn(im, b.post_a[k]);
        } else if (b.post_kind[k] == 1) {
            float f = __fsub_rn(1.0f, __fmul_rn(b.post_a[k], __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im))));
            re = __fmul_rn(re, f);
            im = __fmul_rn(im, f);
        } else {
            float fs = b.post_a[k], lsb = b.post_b[k];
            float xr = re < -fs ? -fs : (re > fs ? fs : re);  // f32::clamp
            float xi = im < -fs ? -fs : (im > fs ? fs : im);
            re = __fmul_rn(roundf(__fdiv_rn(xr, lsb)), lsb);
            im = __fmul_rn(roundf(__fdiv_rn(xi, lsb)), lsb);
        }
    }
    return make_float2(re, im);
}

}  // namespace lpk
