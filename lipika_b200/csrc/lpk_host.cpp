// lpk_host.cpp — host side of the backend: the parts of the reference's
// pipeline that feed the fan-out boundary (src/pipeline.rs prepare(),
// generate_band(), the clock stream and the raw c64 writer), rewritten in
// C++ above the kernel-level ABI.
//
// Table construction uses glibc libm with no FMA contraction
// (-ffp-contract=off), as the reference's Rust code does on x86_64 Linux,
// so trajectory grids and signal tables are bit-identical to its own.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lipika_cuda.h"

namespace lpk {
lpk_status fail(lpk_ctx *ctx, lpk_status code, const std::string &msg);  // lpk_abi.cu
}

namespace {

constexpr double kTau = 6.283185307179586476925286766559;
constexpr double kGm = 3.986005e14;                 // src/geometry/kepler.rs:12
constexpr double kEarthRate = 7.2921151467e-5;      // src/geometry/kepler.rs:13
constexpr double kBoltzmann = 1.380649e-23;         // src/channel/mod.rs:301
constexpr double kChipRate = 1023000.0;             // src/signal/ca_code.rs:23
constexpr double kGridDt = 0.01;                    // src/pipeline.rs:62

inline double rad(double deg) { return deg * (M_PI / 180.0); }  // f64::to_radians

// ------------------------------------------------------------------ RNG
// xoshiro256++ with the SplitMix64 seeding of rand_xoshiro's seed_from_u64.
struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        uint64_t x = seed;
        for (auto &w : s) {
            uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            w = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    void long_jump() {
        static const uint64_t J[4] = {0x76e15d3efefdcbbfULL, 0xc5004e441c522fb3ULL, 0x77710069854ee241ULL,
                                      0x39109bb02acbe635ULL};
        uint64_t t[4] = {0, 0, 0, 0};
        for (uint64_t w : J)
            for (int b = 0; b < 64; ++b) {
                if (w & (1ULL << b))
                    for (int i = 0; i < 4; ++i) t[i] ^= s[i];
                next();
            }
        for (int i = 0; i < 4; ++i) s[i] = t[i];
    }
    bool bool_half() { return next() < 0x8000000000000000ULL; }                          // rand 0.8 gen_bool(0.5)
    uint32_t range16() { return (uint32_t)(((uint64_t)(uint32_t)(next() >> 32) * 16ULL) >> 32); }  // gen_range(0..16)
    // Box–Muller standard normal from two 53-bit uniforms (documented
    // sampler; the reference's rand_distr ziggurat stream is not reproduced).
    double normal() {
        double u1 = (double)((next() >> 11) + 1) * 0x1.0p-53;
        double u2 = (double)(next() >> 11) * 0x1.0p-53;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(kTau * u2);
    }
};

// ------------------------------------------------------------------ geometry
void geodetic(double lat_deg, double lon_deg, double h, double out[3]) {  // geometry/ecef.rs:10-20
    const double a = 6378137.0, f = 1.0 / 298.257223563, e2 = f * (2.0 - f);
    double lat = rad(lat_deg), lon = rad(lon_deg);
    double sl = std::sin(lat), cl = std::cos(lat);
    double n = a / std::sqrt(1.0 - e2 * sl * sl);
    out[0] = (n + h) * cl * std::cos(lon);
    out[1] = (n + h) * cl * std::sin(lon);
    out[2] = (n * (1.0 - e2) + h) * sl;
}

void kepler(const lpk_trajectory_cfg &k, double t, double out[3]) {  // geometry/kepler.rs:27-85
    double r = k.semi_major_axis_m;
    double mm = std::sqrt(kGm / (r * r * r));
    double nu = rad(k.true_anomaly_deg_at_epoch) + mm * (t - k.epoch_unix);
    double snu = std::sin(nu), cnu = std::cos(nu);
    double inc = rad(k.inclination_deg), om = rad(k.raan_deg);
    double si = std::sin(inc), ci = std::cos(inc), so = std::sin(om), co = std::cos(om);
    double xp = r * cnu, yp = r * snu;
    double y1 = yp * ci, z1 = yp * si;
    double xe = xp * co - y1 * so, ye = xp * so + y1 * co;
    double th = kEarthRate * (t - k.epoch_unix);
    double s = std::sin(th), c = std::cos(th);
    out[0] = xe * c + ye * s;
    out[1] = -xe * s + ye * c;
    out[2] = z1;
}

bool raw_position(const lpk_trajectory_cfg &t, double tu, double out[3]) {
    switch (t.kind) {
    case LPK_TRAJ_STATIONARY_GEODETIC: geodetic(t.lat_deg, t.lon_deg, t.h_m, out); return true;
    case LPK_TRAJ_STATIONARY_ECEF: out[0] = t.x_m; out[1] = t.y_m; out[2] = t.z_m; return true;
    case LPK_TRAJ_CIRCULAR_KEPLERIAN: kepler(t, tu, out); return true;
    default: return false;
    }
}

bool is_stationary(const lpk_trajectory_cfg &t) {
    return t.kind == LPK_TRAJ_STATIONARY_GEODETIC || t.kind == LPK_TRAJ_STATIONARY_ECEF;
}

// ------------------------------------------------------------------ signals
int elapsed_periods(double elapsed, double rate, int64_t &whole, double &frac) {  // signal/mod.rs:50-69
    double p = elapsed * rate;
    if (!std::isfinite(p) || std::fabs(p) >= 9.0e18) return -1;
    double err = std::fma(elapsed, rate, -p);
    double w = std::floor(p);
    double f = (p - w) + err;
    if (f < 0.0) { w -= 1.0; f += 1.0; }
    else if (f >= 1.0) { w += 1.0; f -= 1.0; }
    whole = (int64_t)w;
    frac = f;
    return 0;
}

int frame_anchor(double render, double signal, double rate, int64_t n, double &epoch_rel, int64_t &off) {
    if (!(rate > 0.0)) return -1;  // FrameAnchor::at, signal/mod.rs:87-101
    int64_t w;
    double f;
    if (elapsed_periods(render - signal, rate, w, f)) return -1;
    epoch_rel = -f / rate;
    int64_t m = n > 1 ? n : 1;
    int64_t r = w % m;
    off = r < 0 ? r + m : r;
    return 0;
}

std::vector<int8_t> gold_code(int prn) {  // IS-GPS-200 G1/G2, signal/ca_code.rs:34-78
    static const uint8_t taps[32][2] = {{2, 6}, {3, 7}, {4, 8}, {5, 9}, {1, 9}, {2, 10}, {1, 8}, {2, 9},
                                        {3, 10}, {2, 3}, {3, 4}, {5, 6}, {6, 7}, {7, 8}, {8, 9}, {9, 10},
                                        {1, 4}, {2, 5}, {3, 6}, {4, 7}, {5, 8}, {6, 9}, {1, 3}, {4, 6},
                                        {5, 7}, {6, 8}, {7, 9}, {8, 10}, {1, 6}, {2, 7}, {3, 8}, {4, 9}};
    uint32_t g1 = 0x3FF, g2 = 0x3FF;  // bit i = register stage i+1
    int a = taps[prn - 1][0] - 1, b = taps[prn - 1][1] - 1;
    std::vector<int8_t> out(1023);
    for (int k = 0; k < 1023; ++k) {
        uint32_t o = ((g1 >> 9) ^ (g2 >> a) ^ (g2 >> b)) & 1u;
        uint32_t f1 = ((g1 >> 2) ^ (g1 >> 9)) & 1u;
        uint32_t f2 = ((g2 >> 1) ^ (g2 >> 2) ^ (g2 >> 5) ^ (g2 >> 7) ^ (g2 >> 8) ^ (g2 >> 9)) & 1u;
        g1 = ((g1 << 1) | f1) & 0x3FF;
        g2 = ((g2 << 1) | f2) & 0x3FF;
        out[k] = (int8_t)(1 - 2 * (int)o);
    }
    return out;
}

float gray(uint8_t b0, uint8_t b1) {  // signal/qam16.rs:20-27
    if (!b0 && !b1) return -3.0f;
    if (!b0 && b1) return -1.0f;
    if (b0 && b1) return 1.0f;
    return 3.0f;
}

// ------------------------------------------------------------------ clock
constexpr double kFlickerRate = 128.0;
constexpr int kFlickerPoles = 20;

struct Flicker {  // clock/mod.rs:55-149
    double alpha[kFlickerPoles], gain[kFlickerPoles], state[kFlickerPoles] = {};
    double scale = 0.0;
    Xoshiro rng{0};
    int64_t frontier = -1;
    double hi = 0.0, lo = 0.0;

    double step(double *st, Xoshiro &r) {
        double y = 0.0;
        for (int j = 0; j < kFlickerPoles; ++j) {
            st[j] = alpha[j] * st[j] + gain[j] * (0.0 + 1.0 * r.normal());
            y += st[j];
        }
        return y;
    }
    Flicker(double floor_v, const Xoshiro &seed) {
        double fhi = kFlickerRate / 2.0;
        for (int j = 0; j < kFlickerPoles; ++j) {
            double f = 1e-4 * std::pow(fhi / 1e-4, (double)j / (double)(kFlickerPoles - 1));
            double a = std::exp(-2.0 * M_PI * f / kFlickerRate);
            alpha[j] = a;
            gain[j] = std::sqrt(1.0 - a * a);
        }
        Xoshiro c = seed;
        c.long_jump();
        double cs[kFlickerPoles] = {};
        for (int i = 0; i < 200000; ++i) step(cs, c);
        const int64_t nc = 1 << 18;
        std::vector<double> d((size_t)nc, 0.0);
        double acc = 0.0;
        for (int64_t i = 1; i < nc; ++i) {
            acc += step(cs, c) / kFlickerRate;
            d[i] = acc;
        }
        const int64_t m = (int64_t)(2.0 * kFlickerRate);
        double tau = (double)m / kFlickerRate, sum = 0.0;
        int64_t cnt = 0;
        for (int64_t i = 0; i + 2 * m < nc; i += m) {
            double x = d[i + 2 * m] - 2.0 * d[i + m] + d[i];
            sum += x * x;
            ++cnt;
        }
        double meas = std::sqrt((sum / (double)(cnt > 1 ? cnt : 1)) / (2.0 * tau * tau));
        if (meas < 1e-30) meas = 1e-30;
        scale = floor_v / meas;
        rng = seed;
        rng.long_jump();
        rng.long_jump();
        for (int i = 0; i < 200000; ++i) step(state, rng);
    }
    double at(double elapsed) {
        double x = (elapsed > 0.0 ? elapsed : 0.0) * kFlickerRate;
        double fl = std::floor(x);
        int64_t m0 = (int64_t)fl;
        double frac = x - (double)m0;
        while (frontier < m0 + 1) {
            lo = hi;
            hi += step(state, rng) * scale / kFlickerRate;
            ++frontier;
        }
        return lo * (1.0 - frac) + hi * frac;
    }
};

}  // namespace

// ClockStream (src/clock/mod.rs:229-347): forward-only Δt(t) generator.
struct lpk_clock {
    double start, rate, c0, y0, step_std;
    bool walk;
    Xoshiro rng;
    int64_t frontier = -1;
    double eps_hi = 0.0, eps_lo = 0.0;
    std::unique_ptr<Flicker> flicker;

    lpk_clock(const lpk_clock_cfg &s, double start_epoch, double master, uint64_t seed)
        : start(start_epoch), rate(master), c0(s.initial_time_offset_s), y0(s.frequency_offset_y0),
          step_std(0.0), walk(s.allan_deviation_1s > 0.0), rng(seed) {
        if (walk) step_std = s.allan_deviation_1s / std::sqrt(master);
        if (s.flicker_floor > 0.0) flicker.reset(new Flicker(s.flicker_floor, rng));
    }
    void advance(int64_t k) {
        while (frontier < k) {
            eps_lo = eps_hi;
            if (walk) eps_hi += 0.0 + step_std * rng.normal();
            ++frontier;
        }
    }
    double det(double e) const { return c0 + y0 * e; }
    double delta_t_at(double t) {
        double e = t - start;
        double x = e * rate;
        if (x <= 0.0) {
            advance(0);
            double fl = flicker ? flicker->at(0.0) : 0.0;
            return eps_hi + fl + det(0.0);
        }
        int64_t k0 = (int64_t)std::floor(x);
        double frac = x - (double)k0;
        advance(k0 + 1);
        double eps = eps_lo * (1.0 - frac) + eps_hi * frac;
        double fl = flicker ? flicker->at(e) : 0.0;
        return eps + fl + det(e);
    }
};

int64_t lpk_clock_flicker_len(double duration_s) {
    if (!(duration_s >= 0.0) || !std::isfinite(duration_s) || duration_s > 1e9) return -1;
    return (int64_t)std::ceil(duration_s * kFlickerRate) + 2;
}

lpk_status lpk_clock_flicker_table(const lpk_clock_cfg *spec, uint64_t seed, double *out, int64_t n) {
    if (!spec || !out || n < 0) return lpk::fail(nullptr, LPK_EINVAL, "NULL spec or output, or n < 0");
    if (!(spec->flicker_floor > 0.0) || !std::isfinite(spec->flicker_floor))
        return lpk::fail(nullptr, LPK_EINVAL, "the clock has no flicker floor");
    // the host stream's flicker, advanced point by point: D[m] after the
    // step that moves its frontier to m (Flicker::advance_to, clock/mod.rs:130-140)
    Flicker f(spec->flicker_floor, Xoshiro(seed));
    for (int64_t m = 0; m < n; ++m) {
        f.hi += f.step(f.state, f.rng) * f.scale / kFlickerRate;
        out[m] = f.hi;
    }
    return LPK_OK;
}

namespace {

struct TxHost {
    lpk_tx_desc desc{};
    std::vector<double> grid;
    std::vector<int8_t> pm, chips, nav;
    std::vector<uint8_t> ook;
    std::vector<lpk_cf32> sym;
    std::vector<double> gate_on;
    double bandwidth_hz = 0.0;
    bool grid_pending = false;  // grid sized, to be filled on the GPU
};

struct RxHost {
    lpk_trajectory_cfg traj{};
    double pos[3] = {0, 0, 0};
    bool stationary = true;
    lpk_clock_cfg clock{};
    std::vector<lpk_band_cfg> bands;
};

}  // namespace

struct lpk_scene {
    lpk_ctx *ctx = nullptr;
    lpk_scene_cfg cfg{};
    std::vector<TxHost> tx;
    std::vector<RxHost> rx;
    std::vector<std::pair<int32_t, int32_t>> work;
    // flicker tracks handed out by lpk_scene_band_desc, per (receiver, clock
    // seed); entries are never erased, so a descriptor's pointer stays valid
    // while the scene lives
    std::mutex flicker_mu;
    std::map<std::pair<int32_t, uint64_t>, std::vector<double>> flicker;
};

namespace {

lpk_status host_fail(lpk_status code, const std::string &msg) { return lpk::fail(nullptr, code, msg); }

double tx_bandwidth(const lpk_transmitter_cfg &t) {  // config/mod.rs:191-193, :260-268
    if (t.has_bandwidth) return t.bandwidth_hz;
    switch (t.kind) {
    case LPK_SIG_CW: return 0.0;
    case LPK_SIG_CA_CODE: return 2.0 * kChipRate;
    default: return 2.0 * t.rate_hz;
    }
}

// Transmitter::from_config + build_signal (src/pipeline.rs:141-253, :311-341).
// device_grid: a circular Keplerian grid is sized here and filled later by
// lpk_kepler_tables (h.grid_pending).
lpk_status build_tx(const lpk_transmitter_cfg &c, const lpk_scene_cfg &scene, TxHost &h, bool device_grid) {
    lpk_tx_desc &d = h.desc;
    memset(&d, 0, sizeof d);
    const double render = scene.epoch_unix;
    if (is_stationary(c.trajectory)) {
        d.traj_kind = LPK_TX_TRAJ_STATIONARY;
        raw_position(c.trajectory, render, d.stationary_ecef);
    } else if (c.trajectory.kind == LPK_TRAJ_CIRCULAR_KEPLERIAN) {
        // PrecomputedTrajectory::sample (geometry/precomputed.rs:180-204)
        double start = render - 0.5;
        double total = scene.duration_s + 2.0 * 0.5;
        int64_t n = (int64_t)std::ceil(total / kGridDt) + 1;
        if (!(n >= 2) || n > (int64_t)1 << 31) return host_fail(LPK_EINVAL, "trajectory grid size out of range");
        h.grid.resize(3 * (size_t)n);
        h.grid_pending = device_grid;
        for (int64_t i = 0; i < n && !device_grid; ++i) {
            double p[3];
            kepler(c.trajectory, start + (double)i * kGridDt, p);
            h.grid[i] = p[0];
            h.grid[n + i] = p[1];
            h.grid[2 * n + i] = p[2];
        }
        d.traj_kind = LPK_TX_TRAJ_PRECOMPUTED;
        d.grid_t0_unix = start;
        d.grid_dt_s = kGridDt;
        d.grid_n = n;
        d.grid_xyz = h.grid.data();
    } else {
        return host_fail(LPK_ENOTSUP, "transmitter trajectory kind not supported (TLE / RINEX)");
    }
    d.sig_kind = c.kind;
    d.carrier_hz = c.carrier_hz;
    d.tx_power_w = std::pow(10.0, c.tx_power_dbw / 10.0);  // pipeline.rs:338
    h.bandwidth_hz = tx_bandwidth(c);
    bool anchored = c.has_signal_epoch || scene.time_base == LPK_TIME_BASE_ABSOLUTE;
    double anchor = c.has_signal_epoch ? c.signal_epoch_unix : scene.default_signal_epoch_unix;
    switch (c.kind) {
    case LPK_SIG_CW:
        d.cw_offset_hz = c.baseband_offset_hz;
        if (anchored) {  // ContinuousWave::anchor_phase (cw.rs:22-34)
            int64_t w;
            double f;
            if (elapsed_periods(render - anchor, c.baseband_offset_hz, w, f))
                return host_fail(LPK_EINVAL, "cw anchor: cycle count not representable");
            d.cw_anchored = 1;
            d.cw_phase0 = kTau * f;
        }
        break;
    case LPK_SIG_BPSK:
    case LPK_SIG_OOK:
    case LPK_SIG_QAM16: {
        if (c.payload_n < 0 || c.sync_n < 0 || (c.sync_n > 0 && !c.sync_word))
            return host_fail(LPK_EINVAL, "bad payload / sync word");
        Xoshiro rng(c.payload_seed);
        if (c.kind == LPK_SIG_BPSK) {  // BpskFrame::random (bpsk.rs:28-42)
            h.pm.reserve((size_t)c.sync_n + (size_t)c.payload_n);
            h.pm.assign(c.sync_word, c.sync_word + c.sync_n);
            for (int64_t i = 0; i < c.payload_n; ++i) h.pm.push_back(rng.bool_half() ? 1 : -1);
            d.n_sym = (int64_t)h.pm.size();
            d.pm_bits = h.pm.data();
        } else if (c.kind == LPK_SIG_OOK) {  // OokFrame::random (ook.rs:27-44)
            for (int i = 0; i < c.sync_n; ++i)
                if (c.sync_word[i] < 0 || c.sync_word[i] > 1)
                    return host_fail(LPK_EINVAL, "ook sync_word entries must be 0 or 1");
            h.ook.reserve((size_t)c.sync_n + (size_t)c.payload_n);
            for (int i = 0; i < c.sync_n; ++i) h.ook.push_back((uint8_t)c.sync_word[i]);
            for (int64_t i = 0; i < c.payload_n; ++i) h.ook.push_back((uint8_t)rng.bool_half());
            d.n_sym = (int64_t)h.ook.size();
            d.ook_bits = h.ook.data();
        } else {  // Qam16Frame::random (qam16.rs:52-80)
            for (int i = 0; i < c.sync_n; ++i)
                if (c.sync_word[i] < 0 || c.sync_word[i] > 1)
                    return host_fail(LPK_EINVAL, "qam16 sync_word entries must be 0 or 1");
            if (c.sync_n % 4) return host_fail(LPK_EINVAL, "qam16 sync_word must hold whole symbols");
            const float scale = 0.31622777f;
            h.sym.reserve((size_t)(c.sync_n / 4) + (size_t)c.payload_n);
            for (int i = 0; i < c.sync_n; i += 4) {
                const int8_t *b = c.sync_word + i;
                h.sym.push_back({gray((uint8_t)b[0], (uint8_t)b[1]) * scale, gray((uint8_t)b[2], (uint8_t)b[3]) * scale});
            }
            lpk_cf32 point[16];  // map_symbol (qam16.rs:32-34) of each 4-bit value, same f32 products
            for (uint32_t v = 0; v < 16; ++v)
                point[v] = {gray((v >> 3) & 1, (v >> 2) & 1) * scale, gray((v >> 1) & 1, v & 1) * scale};
            for (int64_t i = 0; i < c.payload_n; ++i) h.sym.push_back(point[rng.range16()]);
            d.n_sym = (int64_t)h.sym.size();
            d.symbols = h.sym.data();
        }
        d.rate_hz = c.rate_hz;
        d.epoch_rel_s = 0.0;
        if (anchored) {
            d.has_repeat = 1;
            if (frame_anchor(render, anchor, c.rate_hz, d.n_sym, d.epoch_rel_s, d.repeat_from))
                return host_fail(LPK_EINVAL, "frame anchor: symbol count not representable");
        }
        break;
    }
    case LPK_SIG_CA_CODE:
        if (c.prn < 1 || c.prn > 32) return host_fail(LPK_EINVAL, "PRN must be 1..32");
        h.chips = gold_code(c.prn);
        d.chips = h.chips.data();
        if (scene.time_base == LPK_TIME_BASE_SCENE) {
            d.epoch_rel_s = c.ca_epoch_unix - render;
            if (c.nav == LPK_NAV_DUMMY) {
                d.nav_kind = LPK_NAV_DUMMY;
                d.nav_seed = c.nav_seed + (uint64_t)c.prn * 0xD1B54A32D192ED03ULL;
            } else if (c.nav == LPK_NAV_FULL) {
                return host_fail(LPK_ENOTSUP, "ca_code nav = \"full\" (LNAV generation) is not built here");
            } else {
                d.nav_kind = LPK_NAV_OFF;
            }
        } else {
            if (c.nav != LPK_NAV_OFF)
                return host_fail(LPK_EINVAL, "ca_code with navigation data is not supported in a window render");
            int64_t off;
            if (frame_anchor(render, c.ca_epoch_unix, kChipRate / 1023.0, 1, d.epoch_rel_s, off))
                return host_fail(LPK_EINVAL, "ca_code anchor: period count not representable");
            d.nav_kind = LPK_NAV_OFF;
        }
        break;
    default:
        return host_fail(LPK_EINVAL, "unknown signal kind");
    }
    if (c.has_gate) {  // BurstGate::anchored (gate.rs:36-55)
        double per = c.gate_period_s;
        if (!(per > 0.0) || !std::isfinite(per)) return host_fail(LPK_EINVAL, "gate period_s must be positive and finite");
        if (c.gate_n_bursts < 0 || (c.gate_n_bursts > 0 && !c.gate_bursts)) return host_fail(LPK_EINVAL, "bad gate bursts");
        for (int i = 0; i < c.gate_n_bursts; ++i) {
            double off = c.gate_bursts[2 * i], dur = c.gate_bursts[2 * i + 1];
            if (!(off >= 0.0) || !(dur > 0.0) || !(off + dur <= per))
                return host_fail(LPK_EINVAL, "gate burst must lie within one period");
            h.gate_on.push_back(off);
            h.gate_on.push_back(off + dur);
        }
        double phase = render - c.gate_epoch_unix;
        if (!std::isfinite(phase)) return host_fail(LPK_EINVAL, "gate phase must be finite");
        double r = std::fmod(phase, per);
        d.has_gate = 1;
        d.gate_period_s = per;
        d.gate_phase_s = r < 0.0 ? r + std::fabs(per) : r;
        d.gate_n = c.gate_n_bursts;
        d.gate_on = h.gate_on.data();
    }
    return LPK_OK;
}

double band_bandwidth(const lpk_band_cfg &b) { return b.has_bandwidth ? b.bandwidth_hz : b.sample_rate_hz; }

}  // namespace

extern "C" {

lpk_status lpk_clock_new(const lpk_clock_cfg *spec, double start_epoch, double master_rate_hz, uint64_t seed,
                         lpk_clock **out) {
    if (!spec || !out || !(master_rate_hz > 0.0)) return host_fail(LPK_EINVAL, "bad clock arguments");
    *out = new (std::nothrow) lpk_clock(*spec, start_epoch, master_rate_hz, seed);
    return *out ? LPK_OK : LPK_ENOMEM;
}

lpk_status lpk_clock_delta_t(lpk_clock *c, const double *t, int64_t n, double *out) {
    if (!c || (n > 0 && (!t || !out))) return host_fail(LPK_EINVAL, "bad clock query");
    for (int64_t i = 0; i < n; ++i) out[i] = c->delta_t_at(t[i]);
    return LPK_OK;
}

void lpk_clock_free(lpk_clock *c) { delete c; }

lpk_status lpk_scene_prepare(lpk_ctx *ctx, const lpk_scene_cfg *cfg, lpk_scene **out) {
    if (!cfg || !out) return host_fail(LPK_EINVAL, "NULL argument");
    *out = nullptr;
    if (!std::isfinite(cfg->epoch_unix) || !(cfg->duration_s >= 0.0) || !std::isfinite(cfg->duration_s))
        return host_fail(LPK_EINVAL, "scene epoch/duration must be finite (duration >= 0)");
    if (cfg->n_transmitters < 0 || cfg->n_receivers < 0) return host_fail(LPK_EINVAL, "negative counts");
    std::unique_ptr<lpk_scene> s(new lpk_scene());
    s->ctx = ctx;
    s->cfg = *cfg;
    if ((cfg->flags & ~LPK_SCENE_DEVICE_TABLES) != 0) return host_fail(LPK_EINVAL, "unknown scene flags");
    const bool device_grid = (cfg->flags & LPK_SCENE_DEVICE_TABLES) != 0;
    if (device_grid && !ctx) return host_fail(LPK_EINVAL, "LPK_SCENE_DEVICE_TABLES needs a context");
    s->tx.resize((size_t)cfg->n_transmitters);
    {
        // Transmitters are independent (their tables depend only on their own
        // config): built on the host's threads. On failure the lowest failing
        // index is rebuilt alone, so its status and message are reported as a
        // sequential build would report them.
        const int32_t n_tx = cfg->n_transmitters;
        std::vector<lpk_status> status((size_t)n_tx, LPK_OK);
        std::atomic<int32_t> next{0};
        auto work = [&]() {
            for (int32_t i = next++; i < n_tx; i = next++)
                status[(size_t)i] = build_tx(cfg->transmitters[i], *cfg, s->tx[i], device_grid);
        };
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int32_t nt = (int32_t)std::min<unsigned>(hw, (unsigned)std::max(n_tx, 0));
        std::vector<std::thread> pool;
        for (int32_t k = 1; k < nt; ++k) pool.emplace_back(work);
        work();
        for (auto &t : pool) t.join();
        for (int32_t i = 0; i < n_tx; ++i)
            if (status[(size_t)i] != LPK_OK) {
                s->tx[i] = TxHost();
                return build_tx(cfg->transmitters[i], *cfg, s->tx[i], device_grid);
            }
    }
    if (device_grid) {  // every pending grid shares the scene's start, step and length
        std::vector<lpk_kepler_orbit> orbits;
        std::vector<int32_t> which;
        int64_t n = 0;
        double start = 0.0;
        for (int32_t i = 0; i < cfg->n_transmitters; ++i) {
            if (!s->tx[i].grid_pending) continue;
            const lpk_trajectory_cfg &t = cfg->transmitters[i].trajectory;
            orbits.push_back({t.semi_major_axis_m, t.inclination_deg, t.raan_deg, t.true_anomaly_deg_at_epoch,
                              t.epoch_unix});
            which.push_back(i);
            n = s->tx[i].desc.grid_n;
            start = s->tx[i].desc.grid_t0_unix;
        }
        if (!orbits.empty()) {
            std::vector<double> all(orbits.size() * 3 * (size_t)n);
            lpk_status st = lpk_kepler_tables(ctx, orbits.data(), (int32_t)orbits.size(), start, kGridDt, n,
                                              all.data());
            if (st) return st;
            for (size_t j = 0; j < which.size(); ++j) {
                TxHost &h = s->tx[which[j]];
                const size_t len = 3 * (size_t)n;
                std::copy(all.begin() + (ptrdiff_t)(j * len), all.begin() + (ptrdiff_t)((j + 1) * len),
                          h.grid.begin());
                h.grid_pending = false;
            }
        }
    }
    s->rx.resize((size_t)cfg->n_receivers);
    for (int32_t r = 0; r < cfg->n_receivers; ++r) {
        const lpk_receiver_cfg &rc = cfg->receivers[r];
        if (rc.n_bands < 1 || !rc.bands) return host_fail(LPK_EINVAL, "receiver has no bands");
        RxHost &h = s->rx[r];
        h.traj = rc.trajectory;
        h.stationary = is_stationary(rc.trajectory);
        if (!raw_position(rc.trajectory, cfg->epoch_unix, h.pos))
            return host_fail(LPK_ENOTSUP, "receiver trajectory kind not supported (TLE / RINEX)");
        h.clock = rc.clock;
        h.bands.assign(rc.bands, rc.bands + rc.n_bands);
        for (int32_t b = 0; b < rc.n_bands; ++b) {
            if (!(rc.bands[b].sample_rate_hz > 0.0) || !std::isfinite(rc.bands[b].sample_rate_hz))
                return host_fail(LPK_EINVAL, "band sample_rate_hz must be positive");
            s->work.push_back({r, b});
        }
    }
    if (ctx) {
        std::vector<lpk_tx_desc> descs;
        for (auto &t : s->tx) descs.push_back(t.desc);
        lpk_status st = lpk_scene_upload(ctx, descs.data(), (int32_t)descs.size());
        if (st) return st;
    }
    *out = s.release();
    return LPK_OK;
}

void lpk_scene_free(lpk_scene *s) { delete s; }

int32_t lpk_scene_n_work(const lpk_scene *s) { return s ? (int32_t)s->work.size() : 0; }

lpk_status lpk_scene_work(const lpk_scene *s, int32_t w, int32_t *r, int32_t *b) {
    if (!s || w < 0 || w >= (int32_t)s->work.size() || !r || !b) return host_fail(LPK_EINVAL, "bad work index");
    *r = s->work[w].first;
    *b = s->work[w].second;
    return LPK_OK;
}

int64_t lpk_scene_band_samples(const lpk_scene *s, int32_t r, int32_t b) {
    if (!s || r < 0 || r >= (int32_t)s->rx.size() || b < 0 || b >= (int32_t)s->rx[r].bands.size()) return -1;
    return (int64_t)std::llround(s->rx[r].bands[b].sample_rate_hz * s->cfg.duration_s);  // pipeline.rs:856
}

int32_t lpk_scene_band_active(const lpk_scene *s, int32_t r, int32_t b, int32_t *active, int32_t cap) {
    if (!s || r < 0 || r >= (int32_t)s->rx.size() || b < 0 || b >= (int32_t)s->rx[r].bands.size()) return -1;
    const lpk_band_cfg &band = s->rx[r].bands[b];
    int32_t k = 0;
    for (int32_t i = 0; i < (int32_t)s->tx.size(); ++i) {  // bands_overlap, pipeline.rs:70-75, :882-891
        const TxHost &t = s->tx[i];
        if (std::fabs(t.desc.carrier_hz - band.lo_carrier_hz) <= 0.5 * (t.bandwidth_hz + band_bandwidth(band))) {
            if (active && k < cap) active[k] = i;
            ++k;
        }
    }
    return k;
}

lpk_status lpk_scene_tx_desc(const lpk_scene *s, int32_t tx, lpk_tx_desc *out) {
    if (!s || tx < 0 || tx >= (int32_t)s->tx.size() || !out) return host_fail(LPK_EINVAL, "bad transmitter index");
    *out = s->tx[tx].desc;
    return LPK_OK;
}

lpk_status lpk_scene_band_desc(const lpk_scene *s, int32_t r, int32_t b, uint64_t seed_base, int32_t work_idx,
                               lpk_band_desc *d) {
    if (!s || !d || r < 0 || r >= (int32_t)s->rx.size() || b < 0 || b >= (int32_t)s->rx[r].bands.size())
        return host_fail(LPK_EINVAL, "bad band index");
    const RxHost &rx = s->rx[r];
    const lpk_band_cfg &band = rx.bands[b];
    memset(d, 0, sizeof *d);
    d->epoch_unix = s->cfg.epoch_unix;
    d->fs_hz = band.sample_rate_hz;
    d->lo_hz = band.lo_carrier_hz;
    d->noise_power_w = band.has_noise_power ? band.noise_power_w
                                            : kBoltzmann * band.noise_temperature_k * band.sample_rate_hz;
    d->noise_seed = seed_base + (uint64_t)work_idx;  // noise_seed, pipeline.rs:828-830
    for (int k = 0; k < 3; ++k) d->rx_ecef[k] = rx.pos[k];
    if (rx.stationary) {
        d->rx_kind = LPK_RX_STATIONARY;
    } else if (rx.traj.kind == LPK_TRAJ_CIRCULAR_KEPLERIAN) {  // positioned on the device per sample
        d->rx_kind = LPK_RX_KEPLER;
        d->rx_orbit = {rx.traj.semi_major_axis_m, rx.traj.inclination_deg, rx.traj.raan_deg,
                       rx.traj.true_anomaly_deg_at_epoch, rx.traj.epoch_unix};
    } else {
        d->rx_kind = LPK_RX_PER_SAMPLE;
    }
    bool random_clock = rx.clock.allan_deviation_1s > 0.0 || rx.clock.flicker_floor > 0.0;
    d->clock_mode = random_clock ? LPK_CLOCK_HOST : LPK_CLOCK_DETERMINISTIC;
    d->clock_offset_s = rx.clock.initial_time_offset_s;
    d->clock_y0 = rx.clock.frequency_offset_y0;
    d->clock_allan_1s = rx.clock.allan_deviation_1s;
    double master = 0.0;
    for (const auto &bb : rx.bands) master = std::fmax(master, bb.sample_rate_hz);
    d->clock_master_rate_hz = master;
    d->clock_seed = seed_base + 0xC10C000000000000ULL + (uint64_t)r;  // clock_seed, pipeline.rs:825-827
    if (band.has_frontend) {  // RxChain::from_config, rx/mod.rs:117-137
        const lpk_frontend_cfg &fe = band.frontend;
        if (fe.has_antenna) {
            d->has_antenna = 1;
            d->has_cutoff = fe.has_cutoff;
            d->ant_peak_dbi = fe.peak_dbi;
            d->ant_horizon_dbi = fe.horizon_dbi;
            d->ant_fb_db = fe.fb_db;
            d->ant_cutoff_deg = fe.cutoff_deg;
        }
        if (fe.has_gain) d->post[d->n_post++] = {LPK_POST_GAIN, 0, fe.gain_db};
        if (fe.has_nonlinearity)
            d->post[d->n_post++] = {LPK_POST_NONLINEARITY, 0, std::pow(10.0, (fe.iip3_dbm - 30.0) / 10.0)};
        if (fe.has_adc) d->post[d->n_post++] = {LPK_POST_ADC, fe.adc_bits, fe.adc_full_scale_v};
    }
    d->solver = LPK_SOLVER_REFERENCE;
    if (rx.clock.flicker_floor > 0.0) {  // the scene's flicker track of this receiver clock
        lpk_scene *ms = const_cast<lpk_scene *>(s);
        std::lock_guard<std::mutex> lk(ms->flicker_mu);
        std::vector<double> &tab = ms->flicker[{r, d->clock_seed}];
        if (tab.empty()) {
            const int64_t len = lpk_clock_flicker_len(s->cfg.duration_s);
            if (len < 2) return host_fail(LPK_EINVAL, "scene duration out of range for the flicker track");
            tab.resize((size_t)len);
            lpk_status st = lpk_clock_flicker_table(&rx.clock, d->clock_seed, tab.data(), len);
            if (st) {
                tab.clear();
                return st;
            }
        }
        d->flicker_delta_s = tab.data();
        d->flicker_n = (int64_t)tab.size();
    }
    return LPK_OK;
}

namespace {
// A device clock for a band whose descriptor has a random (host-stream)
// clock: the white-FM walk on the device when the clock has one, the flicker
// track (if any) through the descriptor, the deterministic part otherwise.
void use_device_clock(lpk_band_desc &d, const lpk_clock_cfg &clk) {
    if (d.clock_mode != LPK_CLOCK_HOST) return;
    d.clock_mode = clk.allan_deviation_1s > 0.0 ? LPK_CLOCK_DEVICE_WALK : LPK_CLOCK_DETERMINISTIC;
}
}  // namespace

lpk_status lpk_generate_band(lpk_scene *s, int32_t r, int32_t b, uint64_t seed_base, int32_t work_idx,
                             int64_t chunk_samples, int32_t flags, lpk_sink_fn sink, void *user,
                             lpk_band_result *res) {
    if (!s || !sink) return host_fail(LPK_EINVAL, "NULL scene or sink");
    if (!s->ctx) return host_fail(LPK_EINVAL, "scene was prepared without a context");
    lpk_band_desc d;
    lpk_status st = lpk_scene_band_desc(s, r, b, seed_base, work_idx, &d);
    if (st) return st;
    if (!(flags & LPK_NOISE_ON)) d.noise_power_w = 0.0;
    if (flags & LPK_GEN_SPLIT) d.solver = LPK_SOLVER_SPLIT;
    const RxHost &rx = s->rx[r];
    // The device clock covers the white-FM walk and the flicker track; a
    // receiver whose positions the host computes keeps the host stream.
    if ((flags & LPK_GEN_DEVICE_CLOCK) && d.rx_kind != LPK_RX_PER_SAMPLE) use_device_clock(d, rx.clock);
    const int64_t n = lpk_scene_band_samples(s, r, b);
    if (chunk_samples < 1) chunk_samples = 1;
    std::vector<int32_t> active(256);
    int32_t na = lpk_scene_band_active(s, r, b, active.data(), 256);
    if (na > 256) return host_fail(LPK_EINVAL, "more than 256 in-band transmitters");
    lpk_band_result local;
    if (!res) res = &local;
    memset(res, 0, sizeof *res);
    res->n_active = na;
    std::unique_ptr<lpk_clock> clock;
    if (d.clock_mode == LPK_CLOCK_HOST)
        clock.reset(new lpk_clock(rx.clock, 0.0, d.clock_master_rate_hz, d.clock_seed));
    const int64_t cap = chunk_samples < n ? chunk_samples : (n > 0 ? n : 1);
    std::vector<double> t_local, delta, rxpos;
    std::vector<lpk_cf32> out((size_t)cap);
    if (clock) { t_local.resize((size_t)cap); delta.resize((size_t)cap); }
    const bool host_rx = d.rx_kind == LPK_RX_PER_SAMPLE;
    if (host_rx) rxpos.resize(3 * (size_t)cap);
    const double fs = d.fs_hz, epoch = d.epoch_unix;
    int64_t i0 = 0;
    while (i0 < n) {
        int64_t i1 = i0 + chunk_samples < n ? i0 + chunk_samples : n;
        int64_t clen = i1 - i0;
        if (clock) {
            for (int64_t j = 0; j < clen; ++j) t_local[j] = (double)(i0 + j) / fs;  // pipeline.rs:918
            for (int64_t j = 0; j < clen; ++j) delta[j] = clock->delta_t_at(t_local[j]);
        }
        if (host_rx) {  // receiver.position_ecef_batch(epoch + t_utc), pipeline.rs:929-931
            for (int64_t j = 0; j < clen; ++j) {
                double tl = (double)(i0 + j) / fs;
                double dl = clock ? delta[j] : d.clock_offset_s + d.clock_y0 * tl;
                double p[3];
                raw_position(rx.traj, epoch + (tl - dl), p);
                rxpos[j] = p[0];
                rxpos[clen + j] = p[1];
                rxpos[2 * clen + j] = p[2];
            }
        }
        st = lpk_band_chunk(s->ctx, &d, active.data(), na, i0, clen, clock ? delta.data() : nullptr,
                            host_rx ? rxpos.data() : nullptr, out.data(), res->unoccluded);
        if (st) return st;
        int32_t flow = sink(user, out.data(), clen);
        if (flow < 0) return host_fail(LPK_EINVAL, "sink reported an error");
        i0 = i1;
        if (flow == 1 && i0 < n) {
            res->stopped_early = 1;
            break;
        }
    }
    res->n_samples = i0;
    return LPK_OK;
}

namespace {
struct UnitSinkAdapter {
    lpk_unit_sink_fn sink;
    void *user;
    int32_t work_idx;
};
int32_t unit_sink_adapter(void *user, const lpk_cf32 *chunk, int64_t n) {
    UnitSinkAdapter *a = (UnitSinkAdapter *)user;
    return a->sink(a->user, a->work_idx, chunk, n);
}
}  // namespace

lpk_status lpk_generate_scene(lpk_scene *s, uint64_t seed_base, double round_s, int32_t flags, lpk_unit_sink_fn sink,
                              void *user) {
    if (!s || !sink) return host_fail(LPK_EINVAL, "NULL scene or sink");
    if (!s->ctx) return host_fail(LPK_EINVAL, "scene was prepared without a context");
    const int32_t n_work = (int32_t)s->work.size();
    std::vector<lpk_work_unit> units;
    std::vector<int32_t> unit_work;  // work index of each batch unit
    std::vector<std::vector<int32_t>> actives;
    std::vector<int32_t> rest;  // work units rendered one by one
    actives.reserve((size_t)n_work);
    for (int32_t w = 0; w < n_work; ++w) {
        const int32_t r = s->work[w].first, b = s->work[w].second;
        lpk_work_unit u;
        memset(&u, 0, sizeof u);
        lpk_status st = lpk_scene_band_desc(s, r, b, seed_base, w, &u.band);
        if (st) return st;
        if (!(flags & LPK_NOISE_ON)) u.band.noise_power_w = 0.0;
        if (flags & LPK_GEN_SPLIT) u.band.solver = LPK_SOLVER_SPLIT;
        const RxHost &rx = s->rx[r];
        if ((flags & LPK_GEN_DEVICE_CLOCK) && u.band.rx_kind != LPK_RX_PER_SAMPLE) use_device_clock(u.band, rx.clock);
        if (u.band.rx_kind == LPK_RX_PER_SAMPLE || u.band.clock_mode == LPK_CLOCK_HOST) {
            rest.push_back(w);
            continue;
        }
        actives.emplace_back(256);
        int32_t na = lpk_scene_band_active(s, r, b, actives.back().data(), 256);
        if (na > 256) return host_fail(LPK_EINVAL, "more than 256 in-band transmitters");
        u.n_active = na;
        u.n_samples = lpk_scene_band_samples(s, r, b);
        units.push_back(u);
        unit_work.push_back(w);
    }
    for (size_t k = 0; k < units.size(); ++k) units[k].active = actives[k].data();
    if (!units.empty()) {
        if ((int)units.size() > 256) return host_fail(LPK_EINVAL, "more than 256 batched work units");
        lpk_batch *batch = nullptr;
        lpk_status st = lpk_batch_create(s->ctx, units.data(), (int32_t)units.size(), round_s, &batch);
        if (st) return st;
        std::unique_ptr<lpk_batch, void (*)(lpk_batch *)> guard(batch, lpk_batch_destroy);
        const int64_t rounds = lpk_batch_n_rounds(batch);
        if ((flags & LPK_GEN_AUTOTUNE) && rounds > 0 && (st = lpk_batch_autotune(batch, rounds / 2, 2, nullptr)))
            return st;
        struct Map {
            lpk_unit_sink_fn sink;
            void *user;
            const int32_t *work;
        } map{sink, user, unit_work.data()};
        auto fwd = [](void *m, int32_t u, const lpk_cf32 *chunk, int64_t n) -> int32_t {
            Map *mp = (Map *)m;
            return mp->sink(mp->user, mp->work[u], chunk, n);
        };
        if ((st = lpk_batch_render(batch, fwd, &map))) return st;
    }
    for (int32_t w : rest) {
        const int32_t r = s->work[w].first, b = s->work[w].second;
        const int64_t chunk = std::max<int64_t>(1, std::llround(round_s * s->rx[r].bands[b].sample_rate_hz));
        UnitSinkAdapter a{sink, user, w};
        lpk_status st = lpk_generate_band(s, r, b, seed_base, w, chunk, flags & ~LPK_GEN_AUTOTUNE, unit_sink_adapter,
                                          &a, nullptr);
        if (st) return st;
    }
    return LPK_OK;
}

namespace {
struct FileSink {
    FILE *f;
    bool failed = false;
};
int32_t file_sink(void *user, const lpk_cf32 *chunk, int64_t n) {
    FileSink *fs = (FileSink *)user;
    // lpk_cf32 is (f32 re, f32 im) little-endian on x86_64/aarch64: the raw
    // complex64 layout of write_complex64_into (output/mod.rs:78-86).
    if ((int64_t)fwrite(chunk, sizeof(lpk_cf32), (size_t)n, fs->f) != n) {
        fs->failed = true;
        return -1;
    }
    return 0;
}
}  // namespace

lpk_status lpk_generate_band_to_file(lpk_scene *s, int32_t r, int32_t b, uint64_t seed_base, int32_t work_idx,
                                     int64_t chunk_samples, int32_t flags, const char *path,
                                     lpk_band_result *res) {
    if (!path) return host_fail(LPK_EINVAL, "path is NULL");
    FILE *f = fopen(path, "wb");
    if (!f) return host_fail(LPK_EINVAL, std::string("cannot create ") + path + ": " + strerror(errno));
    FileSink fs{f};
    lpk_status st = lpk_generate_band(s, r, b, seed_base, work_idx, chunk_samples, flags, file_sink, &fs, res);
    if (fclose(f) != 0 && !st) st = host_fail(LPK_EINVAL, "closing the IQ file failed");
    return st;
}

lpk_status lpk_generate_scene_to_files(lpk_scene *s, uint64_t seed_base, double round_s, int32_t flags,
                                       const char *const *paths) {
    if (!s || !paths) return host_fail(LPK_EINVAL, "NULL scene or paths");
    const int32_t n_work = (int32_t)s->work.size();
    std::vector<FILE *> files((size_t)n_work, nullptr);
    lpk_status st = LPK_OK;
    for (int32_t w = 0; w < n_work && !st; ++w) {
        if (!paths[w]) st = host_fail(LPK_EINVAL, "a work unit's path is NULL");
        else if (!(files[w] = fopen(paths[w], "wb")))
            st = host_fail(LPK_EINVAL, std::string("cannot create ") + paths[w] + ": " + strerror(errno));
    }
    if (!st) {
        // each chunk is appended from the pinned staging on this thread while
        // the GPU renders the next round
        auto sink = [](void *user, int32_t w, const lpk_cf32 *chunk, int64_t n) -> int32_t {
            FileSink fs{((FILE **)user)[w]};
            return file_sink(&fs, chunk, n);
        };
        st = lpk_generate_scene(s, seed_base, round_s, flags, sink, files.data());
    }
    for (FILE *f : files)
        if (f && fclose(f) != 0 && !st) st = host_fail(LPK_EINVAL, "closing an IQ file failed");
    return st;
}

}  // extern "C"
