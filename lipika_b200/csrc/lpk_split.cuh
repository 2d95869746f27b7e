// lpk_split.cuh — split-precision fan-out: FP64 only where it matters.
//
// The reference's emission solve (two fixed-point iterates, src/channel/
// mod.rs:75-96) is a smooth function of the reception time tu, except for
// two things the split path reproduces explicitly:
//  * the lerp table is piecewise linear in time, so each iterate has a slope
//    kink where its query time crosses a 10 ms grid node: every tile is fitted
//    per segment (pieces A and B) and a sample picks its piece from its own
//    query time;
//  * each iterate queries the trajectory at the absolute time epoch + t,
//    which FP64 rounds to ~238 ns: the reference's delay is a fine staircase.
//    The fits are of the unrounded delay; per sample the exact rounding
//    offset of each query (a TwoSum) times ∂delay/∂t of its segment restores
//    the staircase.
// Per (tile of kSplitTile band samples, transmitter) an anchor thread fits
// delay_i(tu) = c0 + Δ(c1 + Δ c2), Δ = tu - tu0, for both iterates from
// unrounded FP64 solves at three times. Per sample: both query offsets, two
// polynomials, the signal index in FP64 with a guard band (a sample within
// `guard` of a chip / bit / symbol boundary, or within `tie` of a rounding
// tie of the second query, is recomputed with the exact reference path, so
// indices stay bit-exact), the carrier phase in FP64 reduced modulo 2π
// (Cody–Waite), then sin/cos, amplitude and the complex MAC in FP32.
#pragma once

#include "lpk_device.cuh"

namespace lpk {

#ifndef LPK_SPLIT_TILE
#define LPK_SPLIT_TILE 1024
#endif
#ifndef LPK_SPLIT_THREADS
#define LPK_SPLIT_THREADS 256
#endif
constexpr int kSplitTile = LPK_SPLIT_TILE;        // band samples per anchor tile
constexpr int kSplitThreads = LPK_SPLIT_THREADS;  // kSplitTile / kSplitThreads samples per thread
// Tiles are aligned to absolute band-sample indices and fitted over a tu range
// that depends only on the tile and the clock's deterministic trend, widened
// by kSplitMargin; a sample whose tu falls outside takes the exact path. So
// the fit, and every output bit, is independent of how the band is chunked.
constexpr double kSplitMargin = 1e-5;  // s

enum : int32_t { kRecExact = 1, kRecNavConst = 2, kRecGateOff = 4 };

struct __align__(16) AnchorRec {
    double tu0, tu_hi;                // fit range; Δ origin tu0
    double node0, node1;              // absolute query time where piece B starts (first / second iterate)
    double p0a[3], p0b[3];            // first-iterate delay pieces (unrounded query)
    double p1a[3], p1b[3];            // second-iterate delay pieces (unrounded query)
    double k0, k1a, k1b;              // ∂delay/∂(query time) per piece
    double tie;                       // guard on a rounding tie of the second query (s)
    double ulp_q;                     // ulp of the absolute query time
    double tau_if;                    // 2π (f_tx - f_lo)
    double guard;                     // emission-time guard band (s)
    float amp0, amp1;                 // amplitude = amp0 + amp1 Δ
    int32_t flags;
    int32_t nav_pm;                   // constant nav sign of the tile (kRecNavConst)
    int64_t sym_raw0, sym_pos0;       // framed kinds: raw symbol count at the tile start and its frame slot
};

// Lerp position at epoch-relative time t with the segment forced to `lo`
// (linear extrapolation beyond it), without rounding epoch + t: de is
// epoch - t0 of the grid, exact.
__device__ __forceinline__ void pos_unrounded(const DevTx &tx, double t, double de, int64_t lo, double &x,
                                              double &y, double &z) {
    if (tx.traj_kind == 0) { x = tx.sx; y = tx.sy; z = tx.sz; return; }
    double frac = (t + de) / tx.dt - (double)lo;
    double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
    double omf = 1.0 - frac;
    x = a.x * omf + b.x * frac;
    y = a.y * omf + b.y * frac;
    z = a.z * omf + b.z * frac;
}

// Segment of the unrounded query time t (clamped) and whether the
// reference's lerp would clamp there.
__device__ __forceinline__ int64_t seg_unrounded(const DevTx &tx, double t, double de, bool &clamped) {
    if (tx.traj_kind == 0) { clamped = false; return 0; }
    double f = (t + de) / tx.dt;
    int64_t lo = floor_to_i64(f);
    clamped = lo < 0 || lo > tx.grid_n - 2;
    return lo < 0 ? 0 : (lo > tx.grid_n - 2 ? tx.grid_n - 2 : lo);
}

// One unrounded iterate: the delay |R(P(tq)) - O| / c with P on segment lo,
// the Sagnac angle ω (tu - tq); also ∂delay/∂tq along the segment.
__device__ __forceinline__ double iterate_unrounded(const DevTx &tx, double tu, double tq, double de, int64_t lo,
                                                    double ox, double oy, double oz, double inv_c, double *range,
                                                    double *dd_dt) {
    double sx, sy, sz;
    pos_unrounded(tx, tq, de, lo, sx, sy, sz);
    double w = kEarthRate * (tu - tq);
    double dx = sx + w * sy - ox, dy = sy - w * sx - oy, dz = sz - oz;
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (range) *range = r;
    if (dd_dt) {
        double vx = 0.0, vy = 0.0, vz = 0.0;
        if (tx.traj_kind != 0) {
            double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
            vx = (b.x - a.x) / tx.dt; vy = (b.y - a.y) / tx.dt; vz = (b.z - a.z) / tx.dt;
        }
        *dd_dt = ((dx * (vx + w * vy) + dy * (vy - w * vx) + dz * vz) / r) * inv_c;
    }
    return r * inv_c;
}

// Both unrounded iterates at tu; the first iterate uses its natural segment,
// the second is forced to lo1 (lo1 < 0: its natural segment).
__device__ __forceinline__ double solve_unrounded(const DevTx &tx, double tu, double de, int64_t lo1, double ox,
                                                  double oy, double oz, double inv_c, double *d0_out,
                                                  double *range) {
    bool cl;
    double t0 = tu - kEmissionLag;
    double d0 = iterate_unrounded(tx, tu, t0, de, seg_unrounded(tx, t0, de, cl), ox, oy, oz, inv_c, nullptr, nullptr);
    if (d0_out) *d0_out = d0;
    double t1 = tu - d0;
    if (lo1 < 0) lo1 = seg_unrounded(tx, t1, de, cl);
    return iterate_unrounded(tx, tu, t1, de, lo1, ox, oy, oz, inv_c, range, nullptr);
}

// Newton form of the quadratic through (0, v0), (h, v1), (2h, v2).
__device__ __forceinline__ void quad3(double v0, double v1, double v2, double h, double c[3]) {
    if (!(h > 0.0)) { c[0] = v0; c[1] = 0.0; c[2] = 0.0; return; }
    double s1 = (v1 - v0) / h, s2 = (v2 - v1) / h;
    c[2] = (s2 - s1) / (2.0 * h);
    c[1] = s1 - c[2] * h;
    c[0] = v0;
}

__device__ __forceinline__ double poly2(const double c[3], double d) { return fma(d, fma(d, c[2], c[1]), c[0]); }

// Slot of raw symbol count `raw` in a frame (frame_index, signal/mod.rs:109-115),
// reached from a known slot `pos0` of `raw0` without a 64-bit modulo in the
// common case. Returns -1 where the one-shot frame is silent.
__device__ __forceinline__ int64_t frame_slot(const DevTx &tx, int64_t raw, int64_t raw0, int64_t pos0) {
    if (!tx.has_repeat) return (raw >= 0 && raw < tx.n_sym) ? raw : -1;
    if (tx.n_sym <= 0) return -1;
    int64_t p = pos0 + (raw - raw0);
    if (p >= tx.n_sym || p < 0) p = i64_rem_euclid(p, tx.n_sym);
    return p;
}

}  // namespace lpk
