// lpk_split.cuh — split-precision fan-out: FP64 only where it matters.
//
// The reference's emission solve (two fixed-point iterates, src/channel/
// mod.rs:75-96) is a smooth function of the reception time tu, except for
// two things the split path reproduces explicitly:
//  * the lerp table is piecewise linear in time, so each iterate has a slope
//    kink where its query time crosses a 10 ms grid node: every tile is fitted
//    per segment (up to four pieces, i.e. tiles up to three grid steps long)
//    and a sample picks its piece from its own query time;
//  * each iterate queries the trajectory at the absolute time epoch + t,
//    which FP64 rounds to ~238 ns: the reference's delay is a fine staircase.
//    The fits are of the unrounded delay; per sample the exact rounding
//    offset of each query (a TwoSum) times ∂delay/∂t of its segment restores
//    the staircase.
// Per (tile of band samples, transmitter) an anchor thread fits
// delay_i(tu) = c0 + Δ(c1 + Δ c2), Δ = tu - tu0, for both iterates from
// unrounded FP64 solves at three times. Per sample: both query offsets, two
// polynomials, the signal index in FP64 with a guard band (a sample within
// `guard` of a chip / bit / symbol boundary, or within `tie` of a rounding
// tie of the second query, is recomputed with the exact reference path, so
// indices stay bit-exact), the carrier phase in FP64 reduced modulo 2π
// (Cody–Waite), then sin/cos, amplitude and the complex MAC in FP32.
#pragma once

#include <cstddef>

#include "lpk_contrib.cuh"

namespace lpk {

// Compiled launch shapes of the fan-out: (index, band samples per tile,
// threads per block, minimum resident blocks per SM). The minimum-blocks
// bound caps registers (65536 / (threads x blocks)); tile / threads is the
// number of samples each thread carries through the transmitter loop.
#define LPK_SPLIT_VARIANTS(X) \
    X(0, 1024, 256, 3)        \
    X(1, 512, 256, 3)         \
    X(2, 1024, 512, 2)        \
    X(3, 512, 256, 4)         \
    X(4, 1024, 256, 2)        \
    X(5, 1024, 512, 1)
constexpr int kSplitVariants = 6;
constexpr int kSplitNodes = 3;  // grid nodes an iterate's query may cross inside one tile
constexpr int kSplitMaxTile = 1024;
constexpr int kSplitMinTile = 512;
constexpr int kAnchorThreads = 128;  // anchor kernels: records staged in shared memory per block
#ifndef LPK_ANCHOR_MINB
#define LPK_ANCHOR_MINB 5  // anchor blocks per SM (96 registers)
#endif
// Tiles are aligned to absolute band-sample indices and fitted over a tu range
// that depends only on the tile and the clock's deterministic trend, widened
// by kSplitMargin; a sample whose tu falls outside takes the exact path. So
// the fit, and every output bit, is independent of how the band is chunked.
constexpr double kSplitMargin = 1e-5;  // s

// kRecExact: the whole tile takes the exact path; kRecNavVary: a C/A nav bit
// boundary falls inside the tile (otherwise nav_pm holds the tile's sign);
// kRecGateOff: the transmitter is silent over the whole tile (gate off, or
// an empty frame), so it adds nothing.
// kRecCaWide: the C/A code phase of the tile spans too many chips for the
// tile-relative chip index (the general modulo path is taken).
enum : int32_t { kRecExact = 1, kRecNavVary = 2, kRecGateOff = 4, kRecCaWide = 8 };

struct __align__(16) AnchorRec {
    // Read by the fast pass for every (sample, transmitter): the first 144
    // bytes, in adjacent 16-byte pairs:
    double p0[3];                     // first-iterate delay, piece 0 (unrounded query)
    double p1[3];                     // second-iterate delay, piece 0
    double k0, k1;                    // ∂delay/∂(query time): first iterate; second iterate, piece 0
    double hm;                        // a second query's rounding offset below hm is not within the
                                      // tie guard of a rounding midpoint: half its ulp less the guard
                                      // (exact: both powers of two; the guard off gives half an ulp + 1)
    double tau_if;                    // 2π (f_tx - f_lo)
    double nts;                       // -2π f_tx (the transmitter's)
    double guard;                     // emission-time guard band (s)
    double chip_base;                 // C/A and framed kinds: 1.5 x 2^52 - f0, f0 a whole chip / symbol
                                      // count at or below the tile's first one (floor(x) + chip_base
                                      // holds floor(x) - f0 in its low 32 bits, exactly)
    double epoch_rel;                 // the transmitter's symbol / chip epoch (scene-epoch relative)
    float amp0, amp1;                 // amplitude = amp0 + amp1 Δ
    int32_t flags;
    int32_t chip_m0;                  // C/A: f0 mod 1023; framed kinds: the frame slot of count f0
                                      // (repeating frame) or f0 itself (one-shot frame)
    int32_t nav_pm;                   // nav sign of the tile (1 with nav off; unused with kRecNavVary)
    int32_t n_nodes;                  // most grid nodes either iterate crosses in the tile
    int32_t sym_lo, sym_hi;           // framed kinds, one-shot frame: the symbols f0 + m of the frame
                                      // are those with m in [sym_lo, sym_hi)
    // Read once per tile, or by the multi-piece passes only:
    double tu0, tu_hi;                // fit range; Δ origin tu0
    // An iterate's query crosses up to kSplitNodes grid nodes inside a tile
    // (a tile up to 3 grid steps long): piece q >= 1 starts at the q-th node
    // (absolute query time, kSplitInf when absent). Pieces 0-1 live here,
    // pieces 2-3 of a tile with n_nodes > 1 in its AnchorExt.
    double node0, node1;              // first node of each iterate
    double p0b[3], p1b[3];            // piece 1 of each iterate
    double k1b;                       // second-iterate slope of piece 1
    // A receiver on an orbit: ∂delay/∂(receiver query time) of the first and
    // second iterate at the tile's fit origin (their changes over the tile,
    // krx1b / krx2b, are in the tile's AnchorExt); they carry the rounding of
    // the receiver's query epoch + tu into the delay.
    float krx1a, krx2a;
};
static_assert(sizeof(AnchorRec) % 16 == 0, "AnchorRec arrays must keep 16-byte alignment");
static_assert(sizeof(AnchorRec) == 240, "a bigger record costs the anchor kernels an SM's worth of occupancy");
static_assert(offsetof(AnchorRec, tu0) == 144 && offsetof(AnchorRec, amp0) == 112,
              "the fast pass's fields fill the record's first 144 bytes");

// Pieces 2-3 of a tile whose iterates cross more than one grid node (low
// sample rates): read from global memory by the multi-node pass only.
struct __align__(16) AnchorExt {
    double node0[2], node1[2];        // second and third nodes
    double p0[2][3], p1[2][3];        // pieces 2-3
    double k1[2];
    float krx1b, krx2b;               // receiver on an orbit: d(krx1a, krx2a)/dΔ (written for every such tile)
    double reserved;
};

// Lerp position at epoch-relative time t with the segment forced to `lo`
// (linear extrapolation beyond it), without rounding epoch + t: de is
// epoch - t0 of the grid, exact. The fraction scales by 1/dt: a smooth
// function of t either way, which is all the fits and the converged solve
// need (the reference's own query keeps its division, solve_reference).
__device__ __forceinline__ void pos_unrounded(const DevTx &tx, double t, double de, int64_t lo, double &x,
                                              double &y, double &z) {
    if (tx.traj_kind == 0) { x = tx.sx; y = tx.sy; z = tx.sz; return; }
    double frac = (t + de) * tx.inv_dt - (double)lo;
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
    double f = (t + de) * tx.inv_dt;
    int64_t lo = floor_to_i64(f);
    clamped = lo < 0 || lo > tx.grid_n - 2;
    return lo < 0 ? 0 : (lo > tx.grid_n - 2 ? tx.grid_n - 2 : lo);
}

// One unrounded iterate: the delay |R(P(tq)) - O| / c with P on segment lo,
// the Sagnac angle ω (tu - tq); also ∂delay/∂tq along the segment.
__device__ __forceinline__ double iterate_unrounded(const DevTx &tx, double tu, double tq, double de, int64_t lo,
                                                    double ox, double oy, double oz, double inv_c, double *range,
                                                    double *dd_dt, double *los = nullptr) {
    double sx, sy, sz;
    pos_unrounded(tx, tq, de, lo, sx, sy, sz);
    double w = kEarthRate * (tu - tq);
    double dx = sx + w * sy - ox, dy = sy - w * sx - oy, dz = sz - oz;
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (range) *range = r;
    if (los) {  // unit line of sight, receiver to source
        los[0] = dx / r;
        los[1] = dy / r;
        los[2] = dz / r;
    }
    if (dd_dt) {
        double vx = 0.0, vy = 0.0, vz = 0.0;
        if (tx.traj_kind != 0) {
            double4 a = load_point(tx.grid + lo), b = load_point(tx.grid + lo + 1);
            vx = (b.x - a.x) * tx.inv_dt; vy = (b.y - a.y) * tx.inv_dt; vz = (b.z - a.z) * tx.inv_dt;
        }
        *dd_dt = ((dx * (vx + w * vy) + dy * (vy - w * vx) + dz * vz) / r) * inv_c;
    }
    return r * inv_c;
}

// Anchor groups. An anchor block fits up to kAnchorGroupTiles consecutive
// tiles (one per lane) of up to kAnchorGroupTx consecutive transmitters
// (one per warp) of one band: each warp works on one transmitter, whose
// record and trajectory points it shares, with the band and the
// transmitters staged in shared memory. Records are stored tile-major, the
// order the fan-out stages them in.
constexpr int kAnchorGroupTiles = 32;
constexpr int kAnchorGroupTx = kAnchorThreads / 32;

// Stage the group's nk transmitters active[0..nk) into stx (all threads).
__device__ __forceinline__ void stage_group_txs(const DevTx *__restrict__ txs, const int32_t *__restrict__ active,
                                                int nk, DevTx *stx) {
    constexpr int wt = (int)(sizeof(DevTx) / 8);
    for (int i = threadIdx.x; i < nk * wt; i += blockDim.x) {
        const int k = i / wt;
        reinterpret_cast<uint64_t *>(stx + k)[i - k * wt] =
            reinterpret_cast<const uint64_t *>(txs + active[k])[i - k * wt];
    }
}

// Store the group's nt x nk records from shared memory (slot l * kAnchorGroupTx
// + j for tile l, transmitter j) to dst[l * n_active + j], coalesced within
// each tile's run (all threads).
__device__ __forceinline__ void store_group(const AnchorRec *srec, AnchorRec *__restrict__ dst, int nt, int nk,
                                            int n_active) {
    constexpr int wr = (int)(sizeof(AnchorRec) / 16);
    const int run = nk * wr;
    for (int i = threadIdx.x; i < nt * run; i += blockDim.x) {
        const int l = i / run, r = i - l * run;
        reinterpret_cast<int4 *>(dst + (int64_t)l * n_active)[r] =
            reinterpret_cast<const int4 *>(srec + l * kAnchorGroupTx)[r];
    }
}

// Newton form of the quadratic through (0, v0), (h, v1), (2h, v2); ih = 1/h.
__device__ __forceinline__ void quad3(double v0, double v1, double v2, double h, double ih, double c[3]) {
    if (!(h > 0.0)) { c[0] = v0; c[1] = 0.0; c[2] = 0.0; return; }
    double s1 = (v1 - v0) * ih, s2 = (v2 - v1) * ih;
    c[2] = (s2 - s1) * (0.5 * ih);
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

constexpr double kSplitInf = __builtin_huge_val();

// Fit one (tile, transmitter): band samples gs..ge (absolute indices) of
// band b. Everything depends only on the tile's absolute position, the
// transmitter and the clock's deterministic trend, never on chunking.
// exact_only: the tile takes the reference-exact path for every sample
// (fan-out under the plain FP64 solver). r: the record (the anchor kernels
// build it in shared memory); x: the tile's extension record, written only
// when an iterate crosses more than one grid node (n_nodes > 1).
//
// The fits need each iterate at three times tu_i = tus + i h. The first
// iterate on its natural segment at those times (d0_i) serves its own fit,
// the second iterate's query times tu_i - d0_i, ∂/∂t at the middle (k0) and
// the nodes; the second iterate per piece at the three times serves its fit,
// k1 (middle) and the ranges at the ends (amplitude). Six evaluations for a
// tile inside one grid segment.
// MOV: the band's receiver is on an orbit (positions and velocities at the
// fit times, line-of-sight slopes for the receiver's query rounding).
template <bool MOV>
__device__ __forceinline__ void fit_anchor(const DevBand &b, const DevTx &tx, int64_t gs, int64_t ge, bool exact_only,
                                           AnchorRec &r, AnchorExt *x) {
    const double tls = (double)gs / b.fs, tle = (double)ge / b.fs;
    const double tus = tls - (b.clock_offset + b.clock_y0 * tls) - kSplitMargin;
    const double h = 0.5 * ((tle - (b.clock_offset + b.clock_y0 * tle) + kSplitMargin) - tus);
    const double tue = tus + 2.0 * h;  // the third fit time, exactly
    const double ih = h > 0.0 ? 1.0 / h : 0.0;
    const double ox = b.rx[0], oy = b.rx[1], oz = b.rx[2];
    const double de = tx.traj_kind != 0 ? b.epoch - tx.t0 : 0.0;
    r.tu0 = tus;
    r.tu_hi = tue;
    r.node0 = r.node1 = kSplitInf;
    r.n_nodes = 0;
    r.tau_if = kTau * (tx.carrier - b.lo);
    r.flags = 0;
    r.nav_pm = 1;
    r.k0 = r.k1 = r.k1b = 0.0;
    for (int i = 0; i < 3; ++i) r.p0[i] = r.p1[i] = r.p0b[i] = r.p1b[i] = 0.0;
    r.chip_base = 0.0;
    r.chip_m0 = 0;
    r.nts = tx.neg_tau_src;
    r.epoch_rel = tx.epoch_rel;
    r.krx1a = r.krx2a = 0.0f;
    if (exact_only) {
        r.amp0 = r.amp1 = 0.0f;
        r.guard = r.hm = 0.0;
        r.sym_lo = r.sym_hi = 0;
        r.flags = kRecExact;
        return;
    }
    const double tu[3] = {tus, tus + h, tue};
    // the receiver at the fit times (unrounded query: orbit time rx_de + tu)
    // and its velocity, which the per-sample receiver-rounding terms need
    double O[3][3], V[3][3], u1[3][3], u2[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if constexpr (MOV) {
            kepler_at(b.rx_orb, b.rx_de + tu[i], O[i][0], O[i][1], O[i][2], V[i]);
            u1[i][0] = u1[i][1] = u1[i][2] = u2[i][0] = u2[i][1] = u2[i][2] = 0.0;
        } else {
            O[i][0] = ox; O[i][1] = oy; O[i][2] = oz;
        }
    }
    double d0[3];
    int64_t l0[3] = {0, 0, 0}, l1[3] = {0, 0, 0};
    bool exact = false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        bool cl = false;
        const double tq = tu[i] - kEmissionLag;
        if (tx.traj_kind != 0) {
            l0[i] = seg_unrounded(tx, tq, de, cl);
            exact |= cl;
        }
        d0[i] = iterate_unrounded(tx, tu[i], tq, de, l0[i], O[i][0], O[i][1], O[i][2], b.inv_c, nullptr,
                                  i == 1 ? &r.k0 : nullptr, MOV ? u1[i] : nullptr);
        if (tx.traj_kind != 0) {
            l1[i] = seg_unrounded(tx, tu[i] - d0[i], de, cl);
            exact |= cl;
        }
    }
    const int64_t n0 = l0[2] - l0[0], n1 = l1[2] - l1[0];
    exact |= n0 < 0 || n0 > kSplitNodes || n1 < 0 || n1 > kSplitNodes;
    if (tx.traj_kind != 0) {
        if (n0 > 0) r.node0 = tx.t0 + (double)(l0[0] + 1) * tx.dt;
        if (n1 > 0) r.node1 = tx.t0 + (double)(l1[0] + 1) * tx.dt;
        r.n_nodes = (int32_t)(n0 > n1 ? n0 : n1);
        if (r.n_nodes > 1) {
            for (int i = 0; i < 2; ++i) {
                x->node0[i] = l0[0] + 1 + i < l0[2] ? tx.t0 + (double)(l0[0] + 2 + i) * tx.dt : kSplitInf;
                x->node1[i] = l1[0] + 1 + i < l1[2] ? tx.t0 + (double)(l1[0] + 2 + i) * tx.dt : kSplitInf;
                x->k1[i] = 0.0;
                for (int j = 0; j < 3; ++j) x->p0[i][j] = x->p1[i][j] = 0.0;
            }
        }
    }
    double rs = 1.0, re = 1.0, te_s = tus, te_e = tue, d1m = 0.0;
    if (!exact) {
        // Each piece fits the iterate with its segment forced (the lerp
        // extrapolated linearly), over the whole tile: smooth, so a
        // quadratic through three points holds it well below 1 ps.
        double v[3];
        for (int64_t p = 0; p <= n0; ++p) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
                v[i] = l0[0] + p == l0[i] ? d0[i]
                                          : iterate_unrounded(tx, tu[i], tu[i] - kEmissionLag, de, l0[0] + p, O[i][0],
                                                              O[i][1], O[i][2], b.inv_c, nullptr, nullptr);
            quad3(v[0], v[1], v[2], h, ih, p == 0 ? r.p0 : (p == 1 ? r.p0b : x->p0[p - 2]));
        }
        for (int64_t p = 0; p <= n1; ++p) {
            double k1 = 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double *range = (i == 0 && p == 0) ? &rs : ((i == 2 && p == n1) ? &re : nullptr);
                v[i] = iterate_unrounded(tx, tu[i], tu[i] - d0[i], de, l1[0] + p, O[i][0], O[i][1], O[i][2], b.inv_c,
                                         range, i == 1 ? &k1 : nullptr,
                                         (MOV && l1[0] + p == l1[i]) ? u2[i] : nullptr);
            }
            if (l1[0] + p == l1[1]) d1m = v[1];  // the second iterate on its natural segment at the middle
            if (p == 0) r.k1 = k1; else if (p == 1) r.k1b = k1; else x->k1[p - 2] = k1;
            quad3(v[0], v[1], v[2], h, ih, p == 0 ? r.p1 : (p == 1 ? r.p1b : x->p1[p - 2]));
        }
        te_s = tus - poly2(r.p1, 0.0);
        te_e = tue - poly2(n1 == 0 ? r.p1 : (n1 == 1 ? r.p1b : x->p1[n1 - 2]), 2.0 * h);
    }
    // a receiver on an orbit: its query epoch + tu rounds like the
    // transmitter queries; krx = -(line of sight · receiver velocity) / c of
    // each iterate, linear over the tile. With an antenna, or where the
    // orbit time of the rounded query would round again, the tile is exact.
    if constexpr (MOV) {
        if (b.has_antenna || !b.rx_split_ok) exact = true;
        double kr[2][2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int i = 2 * e;
            kr[0][e] = -(u1[i][0] * V[i][0] + u1[i][1] * V[i][1] + u1[i][2] * V[i][2]) * b.inv_c;
            kr[1][e] = -(u2[i][0] * V[i][0] + u2[i][1] * V[i][1] + u2[i][2] * V[i][2]) * b.inv_c;
        }
        r.krx1a = (float)kr[0][0];
        x->krx1b = (float)((kr[0][1] - kr[0][0]) * (0.5 * ih));
        r.krx2a = (float)kr[1][0];
        x->krx2b = (float)((kr[1][1] - kr[1][0]) * (0.5 * ih));
    }
    float amp_s = (float)(tx.amp_factor / rs), amp_e = (float)(tx.amp_factor / re);
    if (!exact && b.has_antenna) {
        // Antenna gain (src/channel/mod.rs:190-203) folded into the tile's
        // linear amplitude: the elevation is smooth over a tile; a tile
        // whose elevation range (three points, 1e-3 deg margin) touches a
        // discontinuity of the pattern (0 deg, the cutoff) takes the exact
        // path, one entirely below the cutoff is silent.
        const double te_m = tu[1] - d1m;
        const double el_s = antenna_elevation(tx, b.epoch + te_s, ox, oy, oz);
        const double el_m = antenna_elevation(tx, b.epoch + te_m, ox, oy, oz);
        const double el_e = antenna_elevation(tx, b.epoch + te_e, ox, oy, oz);
        const double lo = fmin(fmin(el_s, el_m), el_e) - 1.0e-3, hi = fmax(fmax(el_s, el_m), el_e) + 1.0e-3;
        if (!(lo == lo) || !(hi == hi) || (lo <= 0.0 && hi >= 0.0) ||
            (b.has_cutoff && lo <= b.ant_cutoff && hi >= b.ant_cutoff)) {
            exact = true;
        } else if (b.has_cutoff && hi < b.ant_cutoff) {
            r.flags |= kRecGateOff;
        } else {
            amp_s = __fmul_rn(amp_s, antenna_pattern(b, el_s));
            amp_e = __fmul_rn(amp_e, antenna_pattern(b, el_e));
        }
    }
    r.amp0 = amp_s;
    r.amp1 = (tue > tus) ? (amp_e - amp_s) / (float)(tue - tus) : 0.0f;
    r.guard = ldexp(16.0, ilogb(fmax(fmax(fabs(te_s), fabs(te_e)), 1.0)) - 52);
    // The second query epoch + t1 rounds to ulp_q; our t1 may differ from the
    // reference's by a few ulp of t1, so a sum within `tie` of a rounding
    // midpoint takes the exact path. When ulp_q is that fine the rounding is
    // immaterial (< 1e-19 s of delay) and the check is off (tie < 0).
    const double ulp_q = ldexp(1.0, ilogb(fmax(fmax(fabs(b.epoch + tus), fabs(b.epoch + tue)), 1e-300)) - 52);
    const double tie = ldexp(8.0, ilogb(fmax(fmax(fabs(tus), fabs(tue)), 1.0)) - 52);
    // A rounding error never exceeds half an ulp, so "|(|err| - half)| > tie"
    // (not within `tie` of a tie) is |err| < half - tie; half and tie are
    // powers of two, so the difference is exact (guard off: always true)
    r.hm = 0.5 * ulp_q - ((8.0 * tie > ulp_q) ? -1.0 : tie);
    r.sym_lo = 0;
    r.sym_hi = 0;
    if (!exact && (tx.sig_kind == kBpsk || tx.sig_kind == kOok || tx.sig_kind == kQam16)) {
        // tile-relative symbol index m = floor(x) - f0 as for the C/A chips;
        // the frame slot then takes 32-bit arithmetic (frame_index,
        // src/signal/mod.rs:109-115)
        const double xs = (te_s - tx.epoch_rel) * tx.rate, xe = (te_e - tx.epoch_rel) * tx.rate;
        const double f0 = floor(xs) - 2.0;
        if (tx.n_sym <= 0) {
            r.flags |= kRecGateOff;  // an empty frame is silent everywhere
        } else if (!(fabs(f0) < 1.0e15) || !(xe - f0 + 2.0 < 1073741824.0) || tx.n_sym >= ((int64_t)1 << 30)) {
            exact = true;
        } else if (!tx.has_repeat && (xe + 2.0 < 0.0 || f0 >= (double)tx.n_sym)) {
            r.flags |= kRecGateOff;  // the tile lies wholly outside the one-shot frame
        } else {
            r.chip_base = 0x1.8p52 - f0;  // exact: |f0| < 1e15 < 2^50
            const int64_t f0i = (int64_t)f0;
            if (tx.has_repeat) {
                r.chip_m0 = (int32_t)i64_rem_euclid((int64_t)((uint64_t)f0i + (uint64_t)tx.repeat_from), tx.n_sym);
                // the per-sample slot wraps at most once: the tile must span
                // fewer symbols than the frame holds
                if (!(xe - f0 + 2.0 < (double)tx.n_sym)) exact = true;
            } else {  // f0 within [-2^30, n_sym) here, so every count below fits 32 bits
                r.chip_m0 = (int32_t)f0i;
                r.sym_lo = (int32_t)(-f0i);
                r.sym_hi = (int32_t)(tx.n_sym - f0i);
            }
        }
    }
    if (!exact && tx.sig_kind == kCa) {  // tile-relative chip index: chip_m0 + (floor(cp) - f0)
        const double cs = (te_s - tx.epoch_rel) * kCaChipRate, ce = (te_e - tx.epoch_rel) * kCaChipRate;
        const double f0 = floor(cs) - 2.0;
        if (!(fabs(f0) < 1.0e15) || !(ce - f0 + 2.0 < 1023.0)) {
            r.flags |= kRecCaWide;
        } else {
            r.chip_base = 0x1.8p52 - f0;  // exact: |f0| < 1e15 < 2^50
            r.chip_m0 = (int32_t)i64_rem_euclid((int64_t)f0, 1023);
        }
    }
    if (!exact && tx.sig_kind == kCa && tx.nav_kind != kNavOff) {
        double ns = (te_s - tx.epoch_rel) * kNavBitRate, ne = (te_e - tx.epoch_rel) * kNavBitRate;
        double fs_ = floor(ns), fe_ = floor(ne), g = r.guard * kNavBitRate;
        if (fs_ == fe_ && ns - fs_ > g && ne - fe_ < 1.0 - g) {
            int64_t bi = (int64_t)fs_;
            int nav = 1;
            if (tx.nav_kind == kNavDummy) nav = nav_bit_pm(tx.nav_seed, bi);
            else if (tx.nav_n > 0) nav = tx.nav_bits[bi < 0 ? 0 : (bi < tx.nav_n ? bi : tx.nav_n - 1)];
            r.nav_pm = nav;
        } else {
            r.flags |= kRecNavVary;
        }
    }
    if (!exact && tx.has_gate) {  // a burst edge inside the tile's emission span -> exact tile
        double span = te_e - te_s, g = r.guard;
        double u = f64_rem_euclid(te_s + tx.gate_phase, tx.gate_period);
        for (int i = 0; i < tx.gate_n && !exact; ++i) {
            double2 on = tx.gate_on[i];
            for (int e = 0; e < 2 && !exact; ++e) {
                double edge = e ? on.y : on.x;
                for (int w = -1; w <= 1; ++w) {
                    double x = edge + w * tx.gate_period;
                    if (x >= u - g && x <= u + span + g) { exact = true; break; }
                }
            }
        }
        if (!exact && !gate_is_on(tx, te_s)) r.flags |= kRecGateOff;
    }
    if (exact) r.flags = kRecExact;
}

// Chunk index of sample s of this thread in a tile starting at chunk index
// `first`: each thread holds pairs of adjacent samples (2·tid, 2·tid+1) in
// every 2·THREADS-sample stride, so a pair shares one AWGN Philox block and
// one 16-byte store.
template <int THREADS>
__device__ __forceinline__ int64_t tile_sample(int64_t first, int s) {
    return first + (int64_t)(s >> 1) * (2 * THREADS) + 2 * (int64_t)threadIdx.x + (s & 1);
}

// Per-sample values shared by every transmitter of the band: the UTC
// reception time tu = t_local - Δt, its offset d from the tile's fit origin,
// the rounding offset q0 of the first trajectory query epoch + (tu - 70 ms),
// and psi = -2π f_lo Δt reduced modulo 2π. The carrier phase
// -2π f (delay + Δt) + 2π (f - f_lo) t_local equals
// -2π f delay + 2π (f - f_lo) tu - 2π f_lo Δt (t_local = tu + Δt), so the
// part that depends on Δt alone is formed once per sample. qr: the rounding
// offset of the receiver's query epoch + tu (a receiver on an orbit only).
struct SampleCtx {
    double tu, d, q0, psi, qr;
};

// t_local and Δt of sample s of this thread (src/pipeline.rs:918-927): the
// values the sample context was built from, recomputed where the exact
// path needs them. Samples outside the chunk take the nearest chunk sample.
template <int THREADS>
__device__ __forceinline__ void sample_clock(const DevBand &b, int64_t first, int s, double rfs, double &tl,
                                             double &dl) {
    const int64_t j = tile_sample<THREADS>(first, s);
    const int64_t jc = j < 0 ? 0 : (j >= b.n ? b.n - 1 : j);
    tl = sample_time((double)(b.i0 + jc), b.fs, rfs);
    dl = band_delta(b, jc, tl);
}

// Per-(tile, transmitter) code paths of the fast pass, chosen outside the
// per-sample loop so that the loop body has no branches.
enum PassKind : int { kPassCa = 0, kPassCaNav, kPassBpsk, kPassOok, kPassQam, kPassCw };

__device__ __forceinline__ int pass_kind(const DevTx &tx, const AnchorRec &r) {
    switch (tx.sig_kind) {
    case kCa: return (r.flags & (kRecNavVary | kRecCaWide)) ? kPassCaNav : kPassCa;
    case kBpsk: return kPassBpsk;
    case kOok: return kPassOok;
    case kQam16: return kPassQam;
    default: return kPassCw;
    }
}

// Baseband at emission time te; clears ok within the guard band of a chip /
// bit / symbol boundary (those samples take the exact path).
template <int K>
__device__ __forceinline__ void split_baseband(const DevTx &tx, const AnchorRec &R, double te, double guard, bool &ok,
                                               float &bre, float &bim) {
    bim = 0.0f;
    if constexpr (K == kPassCa || K == kPassCaNav) {  // ca_code.rs:167-193
        const double dt = __dsub_rn(te, R.epoch_rel);
        const double cp = __dmul_rn(dt, kCaChipRate);
        const double fl = floor(cp), fr = cp - fl, g = guard * kCaChipRate;
        ok &= fr >= g && fr <= 1.0 - g;
        int nav = R.nav_pm;
        if constexpr (K == kPassCaNav) {
            const double nb = __dmul_rn(dt, kNavBitRate), nfl = floor(nb), nfr = nb - nfl, g2 = guard * kNavBitRate;
            ok &= nfr >= g2 && nfr <= 1.0 - g2;
            const int64_t bi = (int64_t)nfl;
            if (tx.nav_kind == kNavDummy) nav = nav_bit_pm(tx.nav_seed, bi);
            else nav = tx.nav_n == 0 ? 1 : tx.nav_bits[bi < 0 ? 0 : (bi < tx.nav_n ? bi : tx.nav_n - 1)];
        }
        int m;
        if constexpr (K == kPassCa) {  // within [0, 2045) for every sample in the fit range
            // fl + chip_base = 1.5 x 2^52 + (fl - f0) exactly (|fl - f0| < 2^51):
            // its low mantissa word is fl - f0, read without a conversion
            m = R.chip_m0 + __double2loint(__dadd_rn(fl, R.chip_base));
            m -= m >= 1023 ? 1023 : 0;
            m = (unsigned)m < 1023u ? m : 0;  // samples outside the fit range are redone exactly
        } else {
            ok &= fabs(fl) <= 1.0e9;
            m = (int)fmax(fmin(fl, 1.0e9), -1.0e9) % 1023;
            m += m < 0 ? 1023 : 0;
        }
        const int chip = ((tx.chip_neg[m >> 5] >> (m & 31)) & 1u) ? -nav : nav;
        bre = (float)chip;
    } else if constexpr (K == kPassBpsk || K == kPassOok || K == kPassQam) {  // frame_index, signal/mod.rs:109-115
        const double f = __dmul_rn(__dsub_rn(te, R.epoch_rel), tx.rate);
        const double fl = floor(f), fr = f - fl, g = guard * tx.rate;
        ok &= fr >= g && fr <= 1.0 - g;
        // m = floor(f) - f0, read from the low word of an exact add (the
        // tile's fit range keeps it small); samples outside the fit range
        // are redone exactly, so only their load has to stay in bounds
        const uint32_t m = (uint32_t)__double2loint(__dadd_rn(fl, R.chip_base));
        const uint32_t n = (uint32_t)tx.n_sym;
        uint32_t p = (uint32_t)R.chip_m0 + m;
        bool on;
        if (tx.has_repeat) {  // uniform over the block
            p -= p >= n ? n : 0u;  // at most one wrap per tile
            on = true;
        } else {
            on = (int32_t)m >= (int32_t)R.sym_lo && (int32_t)m < (int32_t)R.sym_hi;
        }
        p = p < n ? p : 0u;  // keeps the load in bounds; `on` masks the value
        if constexpr (K == kPassBpsk) {
            bre = on ? (float)__ldg(tx.pm + p) : 0.0f;
        } else if constexpr (K == kPassOok) {
            bre = on ? (float)__ldg(tx.ook + p) : 0.0f;
        } else {
            const float2 v = __ldg(tx.sym + p);
            bre = on ? v.x : 0.0f;
            bim = on ? v.y : 0.0f;
        }
    } else {  // CW: the reference rounds ω·t to f32 before an f32 sin/cos (cw.rs:45-50)
        const float ph = tx.cw_anchored
                             ? (float)f64_rem_euclid(__dadd_rn(__dmul_rn(tx.cw_omega, te), tx.cw_phase0), kTau)
                             : (float)__dmul_rn(tx.cw_omega, te);
        sincosf(ph, &bim, &bre);
    }
}

// One transmitter over the thread's S samples (the fast path), without
// branches in the sample loop. A sample within `tie` of a rounding tie of
// the second query, or within the guard band of an index boundary, sets
// its bit in `redo` and is left to the exact path; `fit` has the bits of
// the samples inside the tile's fit range. DBG stores the diagnostics.
// NK: grid nodes inside the tile (0: one piece per iterate; 1: two
// pieces; kSplitNodes: up to four pieces, selected per sample).
// ACC: every fast-path sample is also solved with the reference-exact FP64
// arithmetic (the exact path's solve and phase) and the largest delay and
// carrier-phase differences are kept in acc[0], acc[1]; acc[2] counts the
// fast-path samples compared.
// MOV: a receiver on an orbit: the rounding of its query time enters both
// iterates through the record's krx slopes.
template <int K, bool DBG, int NK, int S, int THREADS, bool ACC = false, bool MOV = false>
__device__ __forceinline__ void split_pass(const DevTx &tx, const AnchorRec &R, const AnchorExt *X, double epoch,
                                           const SampleCtx *sc,
                                           unsigned fit, float *ar, float *ai, unsigned &redo, int64_t first,
                                           double *dbg_phase, double *dbg_temit, double *dbg_delay,
                                           const DevBand *acc_band = nullptr, double *acc = nullptr) {
    // the record's first 144 bytes hold everything read here, in adjacent
    // 16-byte pairs; read from shared memory where used, so the compiler can
    // re-read a value instead of spilling it
    const double k0 = R.k0, hm = R.hm, tau_if = R.tau_if, nts = R.nts, guard = R.guard;
    const float amp0 = R.amp0, amp1 = R.amp1;
    // one piece per iterate (no grid node inside the tile): coefficients in registers
    const double a0 = R.p0[0], a1 = R.p0[1], a2 = R.p0[2];
    const double b0 = R.p1[0], b1 = R.p1[1], b2 = R.p1[2];
    const double ka = R.k1;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const SampleCtx &c = sc[s];
        const double tu = c.tu, d = c.d;
        double t1s, poly1, k1;
        if constexpr (NK > 0) {
            const double q = __dadd_rn(epoch, __dsub_rn(tu, kEmissionLag));
            const int i0 = q >= R.node0;
            const double *p0 = i0 ? R.p0b : R.p0;
            if constexpr (NK > 1) {
                const int j0 = (q >= X->node0[0]) + (q >= X->node0[1]);
                if (j0 > 0) p0 = X->p0[j0 - 1];
            }
            t1s = tu - fma(d, fma(d, p0[2], p0[1]), p0[0]);
        } else {
            t1s = tu - fma(d, fma(d, a2, a1), a0);
        }
        double t1r = fma(-k0, c.q0, t1s);  // the reference's t1
        float df = 0.0f;
        if constexpr (MOV) {
            df = __double2float_rn(d);
            t1r = fma(-(double)__fmaf_rn(X->krx1b, df, R.krx1a), c.qr, t1r);
        }
        const double s1 = __dadd_rn(epoch, t1r);  // its second query
        const double e1 = __dsub_rn(s1, epoch);
        bool ok = fabs(e1 - t1r) < hm;
        if constexpr (NK > 0) {
            const int i1 = s1 >= R.node1;
            const double *p1 = i1 ? R.p1b : R.p1;
            double kk = i1 ? R.k1b : R.k1;
            if constexpr (NK > 1) {
                const int j1 = (s1 >= X->node1[0]) + (s1 >= X->node1[1]);
                if (j1 > 0) {
                    p1 = X->p1[j1 - 1];
                    kk = X->k1[j1 - 1];
                }
            }
            poly1 = fma(d, fma(d, p1[2], p1[1]), p1[0]);
            k1 = kk;
        } else {
            poly1 = fma(d, fma(d, b2, b1), b0);
            k1 = ka;
        }
        double delay = fma(k1, e1 - t1s, poly1);
        if constexpr (MOV) delay = fma((double)__fmaf_rn(X->krx2b, df, R.krx2a), c.qr, delay);
        const double te = tu - delay;
        float bre, bim;
        double rb = 0.0;
        if constexpr (K == kPassCw) {
            // CW (cw.rs:41-52): the reference rounds its baseband phase ω·t to
            // f32 (up to ~1e6 rad over a minute) and takes an f32 sin/cos of
            // that value; here the f32 value is reduced exactly in FP64
            // (Cody–Waite, as below) and folded into the carrier phase, so
            // one sin/cos of the sum replaces the f32 sincos of a large
            // argument and the complex product
            const double pb = (double)(tx.cw_anchored
                                           ? (float)f64_rem_euclid(__dadd_rn(__dmul_rn(tx.cw_omega, te), tx.cw_phase0),
                                                                   kTau)
                                           : (float)__dmul_rn(tx.cw_omega, te));
            const double kb = rint(pb * 0.15915494309189535);
            rb = fma(-kb, 6.2831854820251465, pb);
            rb = fma(-kb, -1.748455600074497e-07, rb);
            bre = 1.0f;
            bim = 0.0f;
        } else {
            split_baseband<K>(tx, R, te, guard, ok, bre, bim);
        }
        // carrier phase −2π f (delay + Δt) + 2π (f − f_lo) t_local, reduced mod 2π
        // (Cody–Waite: 2π to 24 bits, kq·hi exact, then 2π − hi); the f32
        // rounding of the reduced phase is < 1.2e-7 rad, below __sincosf's own error
        const double phase = fma(nts, delay, fma(tau_if, tu, c.psi));
        const double kq = rint(phase * 0.15915494309189535);
        double rr = fma(-kq, 6.2831854820251465, phase);
        rr = fma(-kq, -1.748455600074497e-07, rr);
        double rt = rr;  // the angle of the sin/cos: the carrier phase, plus the baseband phase for CW
        if constexpr (K == kPassCw) {  // both parts in [-π, π]: one wrap brings the sum back
            rt += rb;
            rt += rt > 3.141592653589793 ? -6.283185307179586 : (rt < -3.141592653589793 ? 6.283185307179586 : 0.0);
        }
        float sn, cs;
        __sincosf((float)rt, &sn, &cs);
        // f32 arithmetic spelled out (no contraction choices left to the
        // compiler), so every kernel that inlines this pass agrees bit for bit
        const float amp = __fmaf_rn(amp1, __double2float_rn(d), amp0);
        float vre, vim;
        if constexpr (K == kPassCw) {
            vre = cs;
            vim = sn;
        } else if constexpr (K == kPassQam) {
            vre = __fmaf_rn(bre, cs, __fmul_rn(-bim, sn));
            vim = __fmaf_rn(bre, sn, __fmul_rn(bim, cs));
        } else {  // real baseband (±1 or 0/1)
            vre = __fmul_rn(bre, cs);
            vim = __fmul_rn(bre, sn);
        }
        ok &= (fit >> s) & 1u;
        if constexpr (ACC) {
            if (ok) {
                const DevBand &b = *acc_band;
                double tl, dl;
                sample_clock<THREADS>(b, first, s, __drcp_rn(b.fs), tl, dl);
                double te_ref, r_ref, rox, roy, roz;
                band_rx(b, 0, tu, rox, roy, roz);
                solve_reference(tx, tu, rox, roy, roz, epoch, 2, b.inv_c, te_ref, r_ref);
                const double delay_ref = __dmul_rn(r_ref, b.inv_c);
                const double tif = __dmul_rn(kTau, __dsub_rn(tx.carrier, b.lo));
                const double ph_ref = __dadd_rn(__dmul_rn(tx.neg_tau_src, __dadd_rn(delay_ref, dl)),
                                                __dmul_rn(tif, tl));
                double dp = rr - remainder(ph_ref, kTau);
                dp -= kTau * rint(dp * 0.15915494309189535);
                acc[0] = fmax(acc[0], fabs(delay - delay_ref));
                acc[1] = fmax(acc[1], fabs(dp));
                acc[2] += 1.0;
            }
        }
        ar[s] = ok ? __fmaf_rn(amp, vre, ar[s]) : ar[s];
        ai[s] = ok ? __fmaf_rn(amp, vim, ai[s]) : ai[s];
        redo |= (unsigned)!ok << s;
        if constexpr (DBG) {
            if ((fit >> s) & 1u) {
                const int64_t j = tile_sample<THREADS>(first, s);
                dbg_phase[j] = rr;
                dbg_temit[j] = te;
                dbg_delay[j] = delay;
            }
        }
    }
}

// The exact path's contribution (rare samples and whole exact tiles), out of
// line so the reference arithmetic's registers stay out of the fast loop's.
static __device__ __noinline__ bool exact_contribution(const DevTx &tx, const DevBand &b, double t_local, double tu,
                                                double delta, double ox, double oy, double oz, float &cr, float &ci,
                                                double *ph, double *te, double *rg) {
    return contribution(tx, b, t_local, tu, delta, ox, oy, oz, cr, ci, ph, te, rg);
}

// One tile of S * THREADS band samples starting at chunk index `first`,
// with the tile's transmitters and anchor records staged in shared memory.
// Samples outside [0, b.n) are skipped; the transmitters are summed in
// active-list order and the epilogue (AWGN, receiver chain) is applied.
// UNOCC: report per-transmitter occlusion words (b.unocc_words; antenna
// bands of the per-band path only).
// ACC: accuracy mode (see split_pass): the block's largest delay and phase
// differences go to b.acc_stats[0..1] (atomic max on the bit patterns of
// non-negative doubles), its fast-path and exact-path (sample, transmitter)
// counts are added to b.acc_stats[2..3].
// MOV: the band's receiver is on an orbit (see split_pass); its horizon gate
// is off (an optimisation only: the gated samples are zero either way).
// OOL: the exact path's contribution is an out-of-line call (for fan-outs
// whose exact samples are rare: the reference arithmetic's registers stay
// out of the fast loop's allocation); inline otherwise.
template <int S, int THREADS, bool DBG, bool UNOCC, bool ACC, bool MOV, bool OOL = false>
// xrec: the tile's AnchorExt records in global memory (index k per
// transmitter), read only for tiles that cross more than one grid node.
__device__ __forceinline__ void split_tile(const DevBand &b, const DevTx *stx, const AnchorRec *srec,
                                           const AnchorExt *xrec, int n_active, int64_t first,
                                           float2 *__restrict__ out, double *dbg_phase, double *dbg_temit,
                                           double *dbg_delay) {
    double acc[3] = {0.0, 0.0, 0.0};
    double acc_exact = 0.0;
    SampleCtx sc[S];
    float ar[S], ai[S];
    unsigned live = 0, fit = 0;
    const double tu0 = n_active > 0 ? srec[0].tu0 : 0.0, tu_hi = n_active > 0 ? srec[0].tu_hi : 0.0;
    const double rfs = __drcp_rn(b.fs);
    const double nlo = -kTau * b.lo;  // -2π f_lo
    static_assert(S % 2 == 0, "samples are held in adjacent pairs");
#pragma unroll
    for (int s = 0; s < S; ++s) {
        // A sample outside the chunk takes the values of the nearest chunk
        // sample (in the same tile), so every lane computes on valid inputs;
        // its `live` bit stays clear and nothing of it is stored.
        const int64_t j = tile_sample<THREADS>(first, s);
        const bool lv = j >= 0 && j < b.n;
        const int64_t jc = j < 0 ? 0 : (j >= b.n ? b.n - 1 : j);
        ar[s] = ai[s] = 0.0f;
        const double tl = sample_time((double)(b.i0 + jc), b.fs, rfs);  // src/pipeline.rs:918
        const double dl = band_delta(b, jc, tl);
        const double tu = __dsub_rn(tl, dl);                      // :927
        const double t0q = __dsub_rn(tu, kEmissionLag);
        const double s0 = __dadd_rn(b.epoch, t0q);
        double qr = 0.0;
        if constexpr (MOV) {  // the receiver's query epoch + tu, rounded like s0
            const double sr = __dadd_rn(b.epoch, tu);
            qr = __dsub_rn(__dsub_rn(sr, b.epoch), tu);
        }
        sc[s] = SampleCtx{tu, tu - tu0, __dsub_rn(__dsub_rn(s0, b.epoch), t0q), reduce_2pi(nlo * dl), qr};
        live |= (unsigned)lv << s;
        // the fit range depends only on the tile: the same for every
        // transmitter (the pass sees `fit & live`: a sample outside the
        // chunk is never stored, not even as a diagnostic)
        fit |= (unsigned)(tu >= tu0 && tu <= tu_hi) << s;
    }
    // Horizon gate over the tile's samples (src/channel/horizon.rs): with an
    // antenna cutoff, a transmitter certainly below it for every sample of
    // the tile adds nothing (the exact path would give it zero gain).
    __shared__ double gate_red[96];
    __shared__ unsigned char gate_skip[256];
    const bool hgate = !MOV && b.has_antenna && b.has_cutoff;  // uniform over the block
    if (hgate) {
        double lo = __longlong_as_double(0x7ff0000000000000LL), hi = -lo, r2 = 0.0;
        bool fin = true;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (!((live >> s) & 1u)) continue;
            const double tu = sc[s].tu;
            fin = fin && isfinite(tu);
            lo = fmin(lo, tu);
            hi = fmax(hi, tu);
        }
        block_min_max_and(lo, hi, r2, fin, gate_red);
        for (int k = threadIdx.x; k < n_active; k += blockDim.x) {
            const bool sk =
                fin && certainly_below_cutoff(stx[k], b.epoch, lo, hi, b.rx[0], b.rx[1], b.rx[2], 0.0, b.ant_cutoff);
            gate_skip[k] = sk;
            if (b.gate_stats) {
                atomicAdd(b.gate_stats, 1ull);
                if (sk) atomicAdd(b.gate_stats + 1, 1ull);
            }
        }
        __syncthreads();
    }
    for (int k = 0; k < n_active; ++k) {
        const AnchorRec &R = srec[k];
        if (hgate && gate_skip[k]) continue;
        // gate_off: the transmitter is silent over the tile's fitted span; a
        // sample outside that span (a clock excursion beyond the fit
        // margin) is still evaluated exactly
        const bool gate_off = (R.flags & kRecGateOff) != 0;
        const unsigned outside = live & ~fit;
        if (gate_off && !DBG && outside == 0) continue;
        const DevTx &T = stx[k];
        unsigned redo = gate_off ? (DBG ? live : outside) : live;
        if (!(R.flags & kRecExact) && !gate_off) {
            redo = 0;
            // grid nodes inside the tile, uniform over the block
            const int nk = R.n_nodes > 1 ? kSplitNodes : (R.node0 < kSplitInf || R.node1 < kSplitInf ? 1 : 0);
#define LPK_PASS(KIND)                                                                                           \
    do {                                                                                                         \
        if (nk == 0)                                                                                             \
            split_pass<KIND, DBG, 0, S, THREADS, ACC, MOV>(T, R, xrec + k, b.epoch, sc, fit & live, ar, ai, redo, first,  \
                                                      dbg_phase, dbg_temit, dbg_delay, &b, acc);                  \
        else if (nk == 1)                                                                                        \
            split_pass<KIND, DBG, 1, S, THREADS, ACC, MOV>(T, R, xrec + k, b.epoch, sc, fit & live, ar, ai, redo, first,  \
                                                      dbg_phase, dbg_temit, dbg_delay, &b, acc);                  \
        else                                                                                                     \
            split_pass<KIND, DBG, kSplitNodes, S, THREADS, ACC, MOV>(T, R, xrec + k, b.epoch, sc, fit & live, ar, ai,     \
                                                                redo, first, dbg_phase, dbg_temit, dbg_delay, &b,  \
                                                                acc);                                             \
    } while (0)
            switch (pass_kind(T, R)) {
            case kPassCa: LPK_PASS(kPassCa); break;
            case kPassCaNav: LPK_PASS(kPassCaNav); break;
            case kPassBpsk: LPK_PASS(kPassBpsk); break;
            case kPassOok: LPK_PASS(kPassOok); break;
            case kPassQam: LPK_PASS(kPassQam); break;
            default: LPK_PASS(kPassCw); break;
            }
#undef LPK_PASS
            redo &= live;
            if constexpr (UNOCC) {  // the tile's gain is non-zero throughout its fitted span
                if (__any_sync(0xffffffffu, (fit & live) != 0) && (threadIdx.x & 31) == 0)
                    atomicOr(b.unocc_words + k, 1u);
            }
        }
        if constexpr (ACC) acc_exact += (double)__popc(redo & (gate_off ? outside : live));
        if (redo == 0) continue;
#pragma unroll
        for (int s = 0; s < S; ++s) {  // the exact path: rare samples, or whole exact tiles
            if (!((redo >> s) & 1u)) continue;
            float cr = 0.0f, ci = 0.0f;
            double ph = 0.0, te = 0.0, rg = 0.0, tl, dl;
            sample_clock<THREADS>(b, first, s, rfs, tl, dl);
            double ox = b.rx[0], oy = b.rx[1], oz = b.rx[2];
            if constexpr (MOV) band_rx(b, 0, sc[s].tu, ox, oy, oz);
            bool on;
            if constexpr (OOL) on = exact_contribution(T, b, tl, sc[s].tu, dl, ox, oy, oz, cr, ci, &ph, &te, &rg);
            else on = contribution(T, b, tl, sc[s].tu, dl, ox, oy, oz, cr, ci, &ph, &te, &rg);
            if constexpr (UNOCC) {
                if (on && !gate_off) atomicOr(b.unocc_words + k, 1u);
            } else {
                (void)on;
            }
            if (!gate_off || ((outside >> s) & 1u)) {
                ar[s] = __fadd_rn(ar[s], cr);
                ai[s] = __fadd_rn(ai[s], ci);
            }
            if constexpr (DBG) {
                const int64_t j = tile_sample<THREADS>(first, s);
                dbg_phase[j] = ph;
                dbg_temit[j] = te;
                dbg_delay[j] = rg * b.inv_c;
            }
        }
    }
    if constexpr (ACC) {
        for (int off = 16; off > 0; off >>= 1) {
            acc[0] = fmax(acc[0], __shfl_xor_sync(0xffffffffu, acc[0], off));
            acc[1] = fmax(acc[1], __shfl_xor_sync(0xffffffffu, acc[1], off));
            acc[2] += __shfl_xor_sync(0xffffffffu, acc[2], off);
            acc_exact += __shfl_xor_sync(0xffffffffu, acc_exact, off);
        }
        if ((threadIdx.x & 31) == 0 && b.acc_stats) {
            atomicMax(b.acc_stats + 0, (unsigned long long)__double_as_longlong(acc[0]));
            atomicMax(b.acc_stats + 1, (unsigned long long)__double_as_longlong(acc[1]));
            atomicAdd(b.acc_stats + 2, (unsigned long long)acc[2]);
            atomicAdd(b.acc_stats + 3, (unsigned long long)acc_exact);
        }
    }
#pragma unroll
    for (int s = 0; s < S; s += 2) {  // g = b.i0 + j is even: the pair shares one noise block
        const int64_t j = tile_sample<THREADS>(first, s);
        const unsigned lv = (live >> s) & 3u;
        if (lv == 3u) {
            float2 o0, o1;
            band_epilogue2(b, ar[s], ai[s], ar[s + 1], ai[s + 1], b.i0 + j, o0, o1);
            if ((j & 1) == 0) {
                *reinterpret_cast<float4 *>(out + j) = make_float4(o0.x, o0.y, o1.x, o1.y);
            } else {
                out[j] = o0;
                out[j + 1] = o1;
            }
        } else {
            if (lv & 1u) out[j] = band_epilogue(b, ar[s], ai[s], b.i0 + j);
            if (lv & 2u) out[j + 1] = band_epilogue(b, ar[s + 1], ai[s + 1], b.i0 + j + 1);
        }
    }
}

// Ask for `bytes` (a multiple of 16, from a 16-byte aligned address) of
// global memory to be brought into L2; nothing waits for it (a hint).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Stage the tile's transmitters and anchor records into shared memory
// (8-byte words, all threads of the block).
__device__ __forceinline__ void stage_tile(const DevTx *__restrict__ txs, const int32_t *__restrict__ active,
                                           int n_active, const AnchorRec *__restrict__ recs, DevTx *stx,
                                           AnchorRec *srec, bool load_tx) {
    const int wt = (int)(sizeof(DevTx) / 8), wr = (int)(sizeof(AnchorRec) / 8);
    if (load_tx) {
        for (int k = 0; k < n_active; ++k) {
            const uint64_t *src = reinterpret_cast<const uint64_t *>(txs + active[k]);
            uint64_t *dst = reinterpret_cast<uint64_t *>(stx + k);
            for (int w = threadIdx.x; w < wt; w += blockDim.x) dst[w] = src[w];
        }
    }
    const uint64_t *rsrc = reinterpret_cast<const uint64_t *>(recs);
    uint64_t *rdst = reinterpret_cast<uint64_t *>(srec);
    for (int w = threadIdx.x; w < wr * n_active; w += blockDim.x) rdst[w] = rsrc[w];
}

}  // namespace lpk
