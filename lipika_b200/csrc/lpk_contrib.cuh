// lpk_contrib.cuh — per-sample pieces shared by the fan-out kernels: the
// band-sample clock offset, the receiver position and one transmitter's
// reference-exact contribution.
#pragma once

#include "../../include/lipika_cuda.h"
#include "lpk_device.cuh"
#include "lpk_walk.cuh"

namespace lpk {

// Flicker::delta_at (clock/mod.rs:142-148) on the coarse track: the
// host stream's interpolation, operation for operation. The index is
// clamped to the staged points (a chunk stages every point its samples read).
__device__ __forceinline__ double band_flicker(const DevBand &b, double elapsed) {
    if (!b.flicker) return 0.0;
    const double x = __dmul_rn(elapsed > 0.0 ? elapsed : 0.0, kFlickerRate);
    const double fl = floor(x);
    int64_t m = (int64_t)fl - b.flicker_m0;
    m = m < 0 ? 0 : (m > b.flicker_n - 2 ? b.flicker_n - 2 : m);
    const double frac = __dsub_rn(x, fl);
    return __dadd_rn(__dmul_rn(b.flicker[m], __dsub_rn(1.0, frac)), __dmul_rn(b.flicker[m + 1], frac));
}

__device__ __forceinline__ double band_delta(const DevBand &b, int64_t j, double t_local) {
    if (b.clock_mode == LPK_CLOCK_DETERMINISTIC)  // (ε=0 + flicker) + c + m·t, clock/mod.rs:311-345
        return __dadd_rn(__dadd_rn(0.0, band_flicker(b, t_local)),
                         __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, t_local)));
    if (b.clock_mode == LPK_CLOCK_DEVICE_WALK) {  // ClockStream::delta_t_at, clock/mod.rs:329-346
        double x = __dmul_rn(t_local, b.fm);      // elapsed = t - 0.0
        if (x <= 0.0) {
            double e0 = b.eps[0 - b.eps_k0];
            if (b.eps_carry) e0 = __dadd_rn(b.eps_carry[0], e0);
            return __dadd_rn(__dadd_rn(e0, band_flicker(b, 0.0)),
                             __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, 0.0)));
        }
        int64_t k0 = floor_to_i64(x);
        double frac = __dsub_rn(x, (double)k0);
        double lo = b.eps[k0 - b.eps_k0], hi = b.eps[k0 + 1 - b.eps_k0];
        if (b.eps_carry) {
            lo = __dadd_rn(b.eps_carry[k0 / kWalkBlock], lo);
            hi = __dadd_rn(b.eps_carry[(k0 + 1) / kWalkBlock], hi);
        }
        double eps = __dadd_rn(__dmul_rn(lo, __dsub_rn(1.0, frac)), __dmul_rn(hi, frac));
        return __dadd_rn(__dadd_rn(eps, band_flicker(b, t_local)),
                         __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, t_local)));
    }
    return b.delta[j];
}

// Receiver position of chunk sample j at epoch-relative UTC time tu:
// receiver.trajectory.position_ecef_batch(epoch + t_utc) (src/pipeline.rs:
// 929-931) — a constant, the orbit at the rounded absolute time, or the
// caller's per-sample positions.
__device__ __forceinline__ void band_rx(const DevBand &b, int64_t j, double tu, double &ox, double &oy,
                                        double &oz) {
    if (b.rx_kind == LPK_RX_STATIONARY) { ox = b.rx[0]; oy = b.rx[1]; oz = b.rx[2]; return; }
    if (b.rx_kind == LPK_RX_KEPLER) {
        kepler_at(b.rx_orb, __dsub_rn(__dadd_rn(b.epoch, tu), b.rx_orb.epoch), ox, oy, oz);
        return;
    }
    ox = b.rxpos[j];
    oy = b.rxpos[b.n + j];
    oz = b.rxpos[2 * b.n + j];
}

// One transmitter's contribution at one sample (channel/mod.rs:251-267).
// Returns false when the antenna gain is zero (the sample is skipped and
// the per-transmitter buffer keeps its +0).
__device__ __forceinline__ bool contribution(const DevTx &tx, const DevBand &b, double t_local, double tu,
                                             double delta, double ox, double oy, double oz, float &cr,
                                             float &ci, double *phase_out, double *temit_out,
                                             double *range_out) {
    double t_emit, r;
    solve_reference(tx, tu, ox, oy, oz, b.epoch, 2, b.inv_c, t_emit, r);  // NEWTON_ITERATIONS
    if (temit_out) *temit_out = t_emit;
    if (range_out) *range_out = r;
    float2 bb = baseband(tx, t_emit);
    float g = 1.0f;
    if (b.has_antenna) {
        g = antenna_gain(tx, b, __dadd_rn(b.epoch, t_emit), ox, oy, oz);
        if (g == 0.0f) {
            if (phase_out) *phase_out = 0.0;
            return false;
        }
    }
    double delay = __dmul_rn(r, b.inv_c);
    double tau_if = __dmul_rn(kTau, __dsub_rn(tx.carrier, b.lo));
    double phase = __dadd_rn(__dmul_rn(tx.neg_tau_src, __dadd_rn(delay, delta)), __dmul_rn(tau_if, t_local));
    if (phase_out) *phase_out = remainder(phase, kTau);
    double sp, cp;
    sincos(phase, &sp, &cp);
    float amp = __fmul_rn((float)__ddiv_rn(tx.amp_factor, r), g);
    float cpf = (float)cp, spf = (float)sp;
    cr = __fadd_rn(0.0f, __fmul_rn(amp, __fsub_rn(__fmul_rn(bb.x, cpf), __fmul_rn(bb.y, spf))));
    ci = __fadd_rn(0.0f, __fmul_rn(amp, __fadd_rn(__fmul_rn(bb.x, spf), __fmul_rn(bb.y, cpf))));
    return true;
}

// x reduced modulo 2π into [-π, π] in FP64 (Cody–Waite: 2π to 24 bits, so
// k·hi is exact for |k| < 2^29, then the double nearest 2π − hi): about
// 3e-15 rad of error at |x| ~ 1e9 rad.
__device__ __forceinline__ double reduce_2pi(double x) {
    const double k = rint(x * 0.15915494309189535);
    const double r = fma(-k, 6.2831854820251465, x);
    return fma(-k, -1.748455600074497e-07, r);
}

// One transmitter's contribution at one sample with the all-FP64 arithmetic
// of contribution() and the shortcuts a tuned FP64 kernel takes (within
// tolerance of the reference, not bit-exact): both iterates' table lerps
// scaled by 1/dt instead of divided (position_ecef_batch's form,
// src/geometry/precomputed.rs:136-153); the carrier phase reduced modulo 2π
// in FP64 before one FP64 sincos of the reduced angle (the reference's
// sin/cos of ~1e9 rad take the slow reduction); the CW baseband phase (the
// reference's f32 value, src/signal/cw.rs:41-52) reduced likewise and folded
// into the carrier phase; the amplitude from an f32 division. Returns false
// when the antenna gain is zero.
__device__ __forceinline__ bool contribution_fp64(const DevTx &tx, const DevBand &b, double t_local, double tu,
                                                  double delta, double ox, double oy, double oz, float &cr,
                                                  float &ci) {
    double t = tu - kEmissionLag, r = 0.0;
#pragma unroll
    for (int it = 0; it < 2; ++it) {  // NEWTON_ITERATIONS, src/channel/mod.rs:75-96
        double sx, sy, sz;
        traj_position_batch(tx, b.epoch + t, sx, sy, sz);
        const double wtau = kEarthRate * (tu - t);
        const double dx = (sx + wtau * sy) - ox, dy = (sy - wtau * sx) - oy, dz = sz - oz;
        r = sqrt(dx * dx + dy * dy + dz * dz);
        t = tu - r * b.inv_c;
    }
    float g = 1.0f;
    if (b.has_antenna) {
        g = antenna_gain(tx, b, b.epoch + t, ox, oy, oz);
        if (g == 0.0f) return false;
    }
    float bre = 1.0f, bim = 0.0f;
    double extra = 0.0;
    if (tx.sig_kind == kCw) {
        const float ph = tx.cw_anchored ? (float)f64_rem_euclid(tx.cw_omega * t + tx.cw_phase0, kTau)
                                        : (float)(tx.cw_omega * t);
        extra = reduce_2pi((double)ph);
        if (tx.has_gate && !gate_is_on(tx, t)) bre = 0.0f;
    } else {
        const float2 bb = baseband(tx, t);
        bre = bb.x;
        bim = bb.y;
    }
    const double delay = r * b.inv_c;
    const double phase = tx.neg_tau_src * (delay + delta) + kTau * (tx.carrier - b.lo) * t_local;
    double sp, cp;
    sincos(reduce_2pi(phase) + extra, &sp, &cp);
    const float amp = __fdiv_rn((float)tx.amp_factor, (float)r) * g;
    const float cpf = (float)cp, spf = (float)sp;
    cr = amp * (bre * cpf - bim * spf);
    ci = amp * (bre * spf + bim * cpf);
    return true;
}

// Horizon gate (src/channel/horizon.rs:140-215, certainly_below_cutoff):
// true only if the per-sample path would give every sample of a stretch a
// zero antenna gain for this transmitter — its arrival elevation below the
// cutoff throughout. The stretch is given by its epoch-relative UTC sample
// times [tu_min, tu_max] and a ball (centre, radius) holding every receiver
// position. The bound: every emission time lies in [tu_min - L, tu_max]
// (L a light-time bound), so every source position lies in a ball around
// the position at the middle of that interval whose radius follows from
// the table's speed bound; the elevation of the ball's centre plus the
// angular spread of both balls plus 1e-3 deg must clear the cutoff. Any
// non-finite input answers "not certain".
__device__ __forceinline__ bool certainly_below_cutoff(const DevTx &tx, double epoch, double tu_min, double tu_max,
                                                       double cx, double cy, double cz, double orad,
                                                       double cutoff_deg) {
    const double cn = sqrt(cx * cx + cy * cy + cz * cz);
    if (!isfinite(cn) || !isfinite(orad) || !isfinite(tu_min) || !isfinite(tu_max)) return false;
    double max_speed, max_radius, slack_m;
    if (tx.traj_kind == 0) {
        max_speed = 0.0;
        max_radius = sqrt(tx.sx * tx.sx + tx.sy * tx.sy + tx.sz * tx.sz);
        slack_m = 0.0;
    } else {
        max_speed = tx.max_speed;
        max_radius = tx.max_radius;
        slack_m = 1.0;
    }
    // each iterate's range is at most |S| (1 + ω⊕Δ) + |O| with Δ <= 100 s
    const double light = fmax((1.01 * max_radius + cn + orad) / kSpeedOfLight, kEmissionLag);
    if (!(light <= 100.0)) return false;
    const double t_mag = fmax(fabs(tu_min), fabs(tu_max));
    const double lag = light * (1.0 + 1e-9) + 1e-6 + 1e-12 * t_mag;
    const double t_lo = epoch + (tu_min - lag), t_hi = epoch + tu_max;
    const double t_mid = t_lo + 0.5 * (t_hi - t_lo);
    const double half_span = fmax(t_mid - t_lo, t_hi - t_mid);
    double sx, sy, sz;
    traj_position(tx, t_mid, sx, sy, sz);
    const double srad = max_speed * half_span * (1.0 + 1e-9) + slack_m;
    const double dx = sx - cx, dy = sy - cy, dz = sz - cz;
    const double range = sqrt(dx * dx + dy * dy + dz * dz);
    const double rho = srad + orad;
    if (!(rho < range) || !(orad < cn)) return false;
    const double se = (dx * cx + dy * cy + dz * cz) / (range * cn);
    const double deg = 57.2957795130823208767981548141051703;
    const double el = asin(fmin(fmax(se, -1.0), 1.0)) * deg;
    const double spread = (asin(rho / range) + asin(orad / cn)) * deg;
    return el + spread + 1.0e-3 < cutoff_deg;
}

// Block-wide min / max of two doubles and logical AND of a flag (all
// threads of the block take part; every thread receives the result).
// scratch: 3 x 32 doubles of shared memory.
__device__ __forceinline__ void block_min_max_and(double &lo, double &hi, double &r2, bool &fin, double *scratch) {
    for (int off = 16; off > 0; off >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, off));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, off));
        r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, off));
    }
    fin = __all_sync(0xffffffffu, fin);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) {
        scratch[w] = lo;
        scratch[32 + w] = hi;
        scratch[64 + w] = fin ? r2 : __longlong_as_double(0x7ff8000000000000LL);  // NaN marks "not finite"
    }
    __syncthreads();
    lo = scratch[0];
    hi = scratch[32];
    r2 = scratch[64];
    fin = !isnan(r2);
    for (int k = 1; k < nw; ++k) {
        lo = fmin(lo, scratch[k]);
        hi = fmax(hi, scratch[32 + k]);
        const double v = scratch[64 + k];
        fin = fin && !isnan(v);
        r2 = fmax(r2, v);
    }
    __syncthreads();
}

}  // namespace lpk
