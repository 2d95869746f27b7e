// lpk_contrib.cuh — per-sample pieces shared by the fan-out kernels: the
// band-sample clock offset, the receiver position and one transmitter's
// reference-exact contribution.
#pragma once

#include "../../include/lipika_cuda.h"
#include "lpk_device.cuh"
#include "lpk_walk.cuh"

namespace lpk {

__device__ __forceinline__ double band_delta(const DevBand &b, int64_t j, double t_local) {
    if (b.clock_mode == LPK_CLOCK_DETERMINISTIC)  // (ε=0 + flicker=0) + c + m·t, clock/mod.rs:311-345
        return __dadd_rn(0.0, __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, t_local)));
    if (b.clock_mode == LPK_CLOCK_DEVICE_WALK) {  // ClockStream::delta_t_at, clock/mod.rs:329-346
        double x = __dmul_rn(t_local, b.fm);      // elapsed = t - 0.0
        if (x <= 0.0) {
            double e0 = b.eps[0 - b.eps_k0];
            if (b.eps_carry) e0 = __dadd_rn(b.eps_carry[0], e0);
            return __dadd_rn(__dadd_rn(e0, 0.0), __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, 0.0)));
        }
        int64_t k0 = floor_to_i64(x);
        double frac = __dsub_rn(x, (double)k0);
        double lo = b.eps[k0 - b.eps_k0], hi = b.eps[k0 + 1 - b.eps_k0];
        if (b.eps_carry) {
            lo = __dadd_rn(b.eps_carry[k0 / kWalkBlock], lo);
            hi = __dadd_rn(b.eps_carry[(k0 + 1) / kWalkBlock], hi);
        }
        double eps = __dadd_rn(__dmul_rn(lo, __dsub_rn(1.0, frac)), __dmul_rn(hi, frac));
        return __dadd_rn(__dadd_rn(eps, 0.0), __dadd_rn(b.clock_offset, __dmul_rn(b.clock_y0, t_local)));
    }
    return b.delta[j];
}

__device__ __forceinline__ void band_rx(const DevBand &b, int64_t j, double &ox, double &oy, double &oz) {
    if (b.rx_kind == LPK_RX_STATIONARY) { ox = b.rx[0]; oy = b.rx[1]; oz = b.rx[2]; return; }
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

}  // namespace lpk
