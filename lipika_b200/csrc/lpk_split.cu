// lpk_split.cu — the split-precision fan-out (see lpk_split.cuh for the
// numerical design): k_split_anchor fits each (tile, transmitter), then
// k_band_split evaluates every band sample of the tile against the fits.
#include "lpk_contrib.cuh"
#include "lpk_internal.h"
#include "lpk_split.cuh"

namespace lpk {

namespace {

constexpr double kInf = __builtin_huge_val();

// One thread per (tile, transmitter).
__global__ void __launch_bounds__(128)
k_split_anchor(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active, int32_t n_active,
               int64_t t0, int64_t n_tiles, AnchorRec *__restrict__ recs) {
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n_tiles * n_active) return;
    const int64_t tile = id / n_active;
    const int k = (int)(id - tile * n_active);
    const DevTx &tx = txs[active[k]];
    const int64_t gs = (t0 + tile) * kSplitTile, ge = gs + kSplitTile - 1;  // absolute sample indices
    const double tls = (double)gs / b.fs, tle = (double)ge / b.fs;
    const double tus = tls - (b.clock_offset + b.clock_y0 * tls) - kSplitMargin;
    const double tue = tle - (b.clock_offset + b.clock_y0 * tle) + kSplitMargin;
    const double ox = b.rx[0], oy = b.rx[1], oz = b.rx[2];
    const double h = 0.5 * (tue - tus);
    const double de = tx.traj_kind != 0 ? b.epoch - tx.t0 : 0.0;
    AnchorRec r;
    r.tu0 = tus;
    r.tu_hi = tue;
    r.node0 = r.node1 = kInf;
    r.tau_if = kTau * (tx.carrier - b.lo);
    r.flags = 0;
    r.nav_pm = 1;
    r.k0 = r.k1a = r.k1b = 0.0;
    for (int i = 0; i < 3; ++i) r.p0a[i] = r.p0b[i] = r.p1a[i] = r.p1b[i] = 0.0;
    int64_t lo0s = 0, lo0e = 0, lo1s = 0, lo1e = 0;
    bool exact = false;
    if (tx.traj_kind != 0) {
        bool c1, c2, c3, c4;
        lo0s = seg_unrounded(tx, tus - kEmissionLag, de, c1);
        lo0e = seg_unrounded(tx, tue - kEmissionLag, de, c2);
        double d0s = iterate_unrounded(tx, tus, tus - kEmissionLag, de, lo0s, ox, oy, oz, b.inv_c, nullptr, nullptr);
        double d0e = iterate_unrounded(tx, tue, tue - kEmissionLag, de, lo0e, ox, oy, oz, b.inv_c, nullptr, nullptr);
        lo1s = seg_unrounded(tx, tus - d0s, de, c3);
        lo1e = seg_unrounded(tx, tue - d0e, de, c4);
        exact = c1 || c2 || c3 || c4 || lo0e < lo0s || lo0e > lo0s + 1 || lo1e < lo1s || lo1e > lo1s + 1;
        if (lo0e != lo0s) r.node0 = tx.t0 + (double)lo0e * tx.dt;
        if (lo1e != lo1s) r.node1 = tx.t0 + (double)lo1e * tx.dt;
    }
    double rs = 1.0, re = 1.0, te_s = tus, te_e = tue;
    if (!exact) {
        double v[3];
        for (int piece = 0; piece < 2; ++piece) {
            int64_t lo = piece ? lo0e : lo0s;
            if (piece && lo0e == lo0s) break;
            for (int i = 0; i < 3; ++i) {
                double tu = tus + i * h;
                v[i] = iterate_unrounded(tx, tu, tu - kEmissionLag, de, lo, ox, oy, oz, b.inv_c, nullptr, nullptr);
            }
            quad3(v[0], v[1], v[2], h, piece ? r.p0b : r.p0a);
        }
        for (int piece = 0; piece < 2; ++piece) {
            int64_t lo = piece ? lo1e : lo1s;
            if (piece && lo1e == lo1s) break;
            for (int i = 0; i < 3; ++i)
                v[i] = solve_unrounded(tx, tus + i * h, de, lo, ox, oy, oz, b.inv_c, nullptr, nullptr);
            quad3(v[0], v[1], v[2], h, piece ? r.p1b : r.p1a);
        }
        // ∂delay/∂(query time) of each piece at the tile middle
        bool cl;
        const double mid = tus + h;
        const double tq0 = mid - kEmissionLag;
        double d0m = iterate_unrounded(tx, mid, tq0, de, seg_unrounded(tx, tq0, de, cl), ox, oy, oz, b.inv_c,
                                       nullptr, &r.k0);
        iterate_unrounded(tx, mid, mid - d0m, de, lo1s, ox, oy, oz, b.inv_c, nullptr, &r.k1a);
        r.k1b = r.k1a;
        if (lo1e != lo1s) iterate_unrounded(tx, mid, mid - d0m, de, lo1e, ox, oy, oz, b.inv_c, nullptr, &r.k1b);
        solve_unrounded(tx, tus, de, lo1s, ox, oy, oz, b.inv_c, nullptr, &rs);
        solve_unrounded(tx, tue, de, lo1e, ox, oy, oz, b.inv_c, nullptr, &re);
        te_s = tus - poly2(r.p1a, 0.0);
        te_e = tue - poly2(lo1e != lo1s ? r.p1b : r.p1a, 2.0 * h);
    }
    const float amp_s = (float)(tx.amp_factor / rs), amp_e = (float)(tx.amp_factor / re);
    r.amp0 = amp_s;
    r.amp1 = (tue > tus) ? (amp_e - amp_s) / (float)(tue - tus) : 0.0f;
    r.guard = ldexp(16.0, ilogb(fmax(fmax(fabs(te_s), fabs(te_e)), 1.0)) - 52);
    // The second query epoch + t1 rounds to ulp_q; our t1 may differ from the
    // reference's by a few ulp of t1, so a sum within `tie` of a rounding
    // midpoint takes the exact path. When ulp_q is that fine the rounding is
    // immaterial (< 1e-19 s of delay) and the check is off (tie < 0).
    r.ulp_q = ldexp(1.0, ilogb(fmax(fmax(fabs(b.epoch + tus), fabs(b.epoch + tue)), 1e-300)) - 52);
    const double tie = ldexp(8.0, ilogb(fmax(fmax(fabs(tus), fabs(tue)), 1.0)) - 52);
    r.tie = (8.0 * tie > r.ulp_q) ? -1.0 : tie;
    r.sym_raw0 = 0;
    r.sym_pos0 = 0;
    if (!exact && (tx.sig_kind == kBpsk || tx.sig_kind == kOok || tx.sig_kind == kQam16)) {
        r.sym_raw0 = floor_to_i64((te_s - tx.epoch_rel) * tx.rate);
        r.sym_pos0 = (tx.has_repeat && tx.n_sym > 0)
                         ? i64_rem_euclid((int64_t)((uint64_t)r.sym_raw0 + (uint64_t)tx.repeat_from), tx.n_sym)
                         : r.sym_raw0;
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
            r.flags |= kRecNavConst;
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
    if (exact) r.flags |= kRecExact;
    recs[id] = r;
}

// Per-sample values shared by every transmitter of the band: local and UTC
// reception times, clock offset, and the first trajectory query (epoch + t0
// with t0 = tu - 70 ms, the same for every transmitter) with its rounding.
struct SampleCtx {
    double tl, dl, q0;  // tu = tl - dl and the query epoch + t0 are recomputed where needed
};

constexpr int kKindCa = 0, kKindFramed = 1, kKindCw = 2;

// Baseband of one kind at emission time te; clears ok within the guard band
// of a chip / bit / symbol boundary.
template <int K>
__device__ __forceinline__ void split_baseband(const DevTx &tx, const AnchorRec &R, double te, double guard, bool &ok,
                                               float &bre, float &bim) {
    bre = 0.0f;
    bim = 0.0f;
    if constexpr (K == kKindCa) {
        const double dt = __dsub_rn(te, tx.epoch_rel);
        const double cp = __dmul_rn(dt, kCaChipRate);
        const double fl = floor(cp), fr = cp - fl, g = guard * kCaChipRate;
        ok &= fr >= g && fr <= 1.0 - g && fabs(fl) <= 1.0e9;
        int nav = R.nav_pm;
        if (tx.nav_kind != kNavOff && !(R.flags & kRecNavConst)) {
            const double nb = __dmul_rn(dt, kNavBitRate), nfl = floor(nb), nfr = nb - nfl, g2 = guard * kNavBitRate;
            ok &= nfr >= g2 && nfr <= 1.0 - g2;
            const int64_t bi = (int64_t)nfl;
            if (tx.nav_kind == kNavDummy) nav = nav_bit_pm(tx.nav_seed, bi);
            else nav = tx.nav_n == 0 ? 1 : tx.nav_bits[bi < 0 ? 0 : (bi < tx.nav_n ? bi : tx.nav_n - 1)];
        } else if (tx.nav_kind == kNavOff) {
            nav = 1;
        }
        int m = (int)fmax(fmin(fl, 1.0e9), -1.0e9) % 1023;
        m += m < 0 ? 1023 : 0;
        const int chip = ((tx.chip_neg[m >> 5] >> (m & 31)) & 1u) ? -1 : 1;
        bre = (float)(chip * nav);
    } else if constexpr (K == kKindFramed) {
        const double f = __dmul_rn(__dsub_rn(te, tx.epoch_rel), tx.rate);
        const double fl = floor(f), fr = f - fl, g = guard * tx.rate;
        ok &= fr >= g && fr <= 1.0 - g;
        const int64_t slot = frame_slot(tx, (int64_t)fl, R.sym_raw0, R.sym_pos0);
        if (slot >= 0) {
            if (tx.sig_kind == kBpsk) bre = (float)__ldg(tx.pm + slot);
            else if (tx.sig_kind == kOok) bre = (float)__ldg(tx.ook + slot);
            else { const float2 s = __ldg(tx.sym + slot); bre = s.x; bim = s.y; }
        }
    } else {  // CW: the reference rounds ω·t to f32 before an f32 sin/cos (cw.rs:45-50)
        const float ph = tx.cw_anchored
                             ? (float)f64_rem_euclid(__dadd_rn(__dmul_rn(tx.cw_omega, te), tx.cw_phase0), kTau)
                             : (float)__dmul_rn(tx.cw_omega, te);
        sincosf(ph, &bim, &bre);
    }
}

// One transmitter over the thread's S samples (the split fast path). A
// sample outside the fit, within `tie` of a rounding tie of the second
// query, or within the guard band of an index boundary sets its bit in
// `redo` and is left to the exact path. DBG stores the diagnostics.
template <int K, bool DBG, bool KINK, int S>
__device__ __forceinline__ void split_pass(const DevTx &tx, const AnchorRec &R, double epoch, const SampleCtx *sc,
                                           const bool *live, float *ar, float *ai, unsigned &redo, int64_t first,
                                           double *dbg_phase, double *dbg_temit, double *dbg_delay) {
    const double tu0 = R.tu0, tu_hi = R.tu_hi, node0 = R.node0, node1 = R.node1, k0 = R.k0, tie = R.tie;
    const double half = 0.5 * R.ulp_q, tau_if = R.tau_if, nts = tx.neg_tau_src, guard = R.guard;
    const float amp0 = R.amp0, amp1 = R.amp1;
    // one piece per iterate (no grid node inside the tile): coefficients in registers
    const double a0 = R.p0a[0], a1 = R.p0a[1], a2 = R.p0a[2], b0 = R.p1a[0], b1 = R.p1a[1], b2 = R.p1a[2];
    const double ka = R.k1a;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        if (!live[s]) continue;
        const SampleCtx &c = sc[s];
        const double tu = __dsub_rn(c.tl, c.dl);  // src/pipeline.rs:927
        bool ok = tu >= tu0 && tu <= tu_hi;
        const double d = tu - tu0;
        double t1s, poly1, k1;
        const double *p1 = nullptr;
        if constexpr (KINK) {
            const double *p0 = __dadd_rn(epoch, __dsub_rn(tu, kEmissionLag)) >= node0 ? R.p0b : R.p0a;
            t1s = tu - fma(d, fma(d, p0[2], p0[1]), p0[0]);
        } else {
            t1s = tu - fma(d, fma(d, a2, a1), a0);
        }
        const double t1r = fma(-k0, c.q0, t1s);  // the reference's t1
        const double s1 = __dadd_rn(epoch, t1r);  // its second query
        const double e1 = __dsub_rn(s1, epoch);
        ok &= fabs(fabs(e1 - t1r) - half) > tie;
        if constexpr (KINK) {
            const bool pb = s1 >= node1;
            p1 = pb ? R.p1b : R.p1a;
            poly1 = fma(d, fma(d, p1[2], p1[1]), p1[0]);
            k1 = pb ? R.k1b : R.k1a;
        } else {
            poly1 = fma(d, fma(d, b2, b1), b0);
            k1 = ka;
        }
        (void)p1;
        const double delay = fma(k1, e1 - t1s, poly1);
        const double te = tu - delay;
        float bre, bim;
        split_baseband<K>(tx, R, te, guard, ok, bre, bim);
        // carrier phase −2π f (delay + Δt) + 2π (f − f_lo) t_local, reduced mod 2π
        const double phase = fma(tau_if, c.tl, nts * (delay + c.dl));
        const double kq = rint(phase * 0.15915494309189535);
        double rr = fma(-kq, 6.2831854820251465, phase);  // 2π to 24 bits: kq·hi exact
        rr = fma(-kq, -1.748455600074497e-07, rr);        // 2π − hi
        const float rf = (float)rr, dr = (float)(rr - (double)rf);
        float sn, cs;
        __sincosf(rf, &sn, &cs);
        const float sc2 = fmaf(dr, cs, sn), cc2 = fmaf(-dr, sn, cs);
        const float amp = fmaf(amp1, (float)d, amp0);
        if (ok) {
            ar[s] = fmaf(amp, bre * cc2 - bim * sc2, ar[s]);
            ai[s] = fmaf(amp, bre * sc2 + bim * cc2, ai[s]);
        } else {
            redo |= 1u << s;
        }
        if constexpr (DBG) {
            const int64_t j = first + s * kSplitThreads + threadIdx.x;
            dbg_phase[j] = rr;
            dbg_temit[j] = te;
            dbg_delay[j] = delay;
        }
    }
}

template <bool DBG>
// At least 3 resident blocks per SM (<= 80 registers): measured on the
// dual-band scene, occupancy outweighs the few register spills it costs
// (1 block/SM unconstrained: 5.7e10 tx·rx/s; 3 blocks: 1.05e11).
#ifndef LPK_SPLIT_MINB
#define LPK_SPLIT_MINB 3
#endif
__global__ void __launch_bounds__(kSplitThreads, LPK_SPLIT_MINB)
k_band_split(const DevBand b, const DevTx *__restrict__ txs, const int32_t *__restrict__ active, int32_t n_active,
             int64_t t0, const AnchorRec *__restrict__ recs, float2 *__restrict__ out, double *dbg_phase,
             double *dbg_temit, double *dbg_delay) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DevTx *stx = reinterpret_cast<DevTx *>(smem_raw);
    AnchorRec *srec = reinterpret_cast<AnchorRec *>(smem_raw + sizeof(DevTx) * (size_t)n_active);
    const int64_t tile = blockIdx.x;
    const int64_t first = (t0 + tile) * kSplitTile - b.i0;  // chunk index of the tile's first sample
    {
        const int wt = (int)(sizeof(DevTx) / 8), wr = (int)(sizeof(AnchorRec) / 8);
        for (int k = 0; k < n_active; ++k) {
            const uint64_t *src = reinterpret_cast<const uint64_t *>(txs + active[k]);
            uint64_t *dst = reinterpret_cast<uint64_t *>(stx + k);
            for (int w = threadIdx.x; w < wt; w += blockDim.x) dst[w] = src[w];
        }
        const uint64_t *rsrc = reinterpret_cast<const uint64_t *>(recs + tile * n_active);
        uint64_t *rdst = reinterpret_cast<uint64_t *>(srec);
        for (int w = threadIdx.x; w < wr * n_active; w += blockDim.x) rdst[w] = rsrc[w];
    }
    __syncthreads();
    constexpr int S = kSplitTile / kSplitThreads;
    SampleCtx sc[S];
    float ar[S], ai[S];
    bool live[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int64_t j = first + s * kSplitThreads + threadIdx.x;
        live[s] = j >= 0 && j < b.n;
        ar[s] = ai[s] = 0.0f;
        sc[s] = SampleCtx{0.0, 0.0, 0.0};
        if (live[s]) {
            const double tl = __ddiv_rn((double)(b.i0 + j), b.fs);  // src/pipeline.rs:918
            const double dl = band_delta(b, j, tl);
            const double tu = __dsub_rn(tl, dl);                     // :927
            const double t0q = __dsub_rn(tu, kEmissionLag);
            const double s0 = __dadd_rn(b.epoch, t0q);
            sc[s] = SampleCtx{tl, dl, __dsub_rn(__dsub_rn(s0, b.epoch), t0q)};
        }
    }
    for (int k = 0; k < n_active; ++k) {
        const AnchorRec &R = srec[k];
        const bool gate_off = (R.flags & kRecGateOff) != 0;
        if (gate_off && !DBG) continue;
        const DevTx &T = stx[k];
        unsigned redo = (1u << S) - 1u;
        if (!(R.flags & kRecExact) && !gate_off) {
            redo = 0;
            const bool kink = R.node0 < kInf || R.node1 < kInf;  // warp-uniform
#define LPK_PASS(KIND, KNK) \
    split_pass<KIND, DBG, KNK, S>(T, R, b.epoch, sc, live, ar, ai, redo, first, dbg_phase, dbg_temit, dbg_delay)
            if (T.sig_kind == kCa) {
                if (kink) LPK_PASS(kKindCa, true); else LPK_PASS(kKindCa, false);
            } else if (T.sig_kind == kCw) {
                if (kink) LPK_PASS(kKindCw, true); else LPK_PASS(kKindCw, false);
            } else {
                if (kink) LPK_PASS(kKindFramed, true); else LPK_PASS(kKindFramed, false);
            }
#undef LPK_PASS
        }
        if (redo == 0) continue;
#pragma unroll
        for (int s = 0; s < S; ++s) {  // the exact path: rare samples, or whole exact tiles
            if (!((redo >> s) & 1u) || !live[s]) continue;
            float cr = 0.0f, ci = 0.0f;
            double ph = 0.0, te = 0.0, rg = 0.0;
            contribution(T, b, sc[s].tl, __dsub_rn(sc[s].tl, sc[s].dl), sc[s].dl, b.rx[0], b.rx[1], b.rx[2], cr, ci, &ph, &te, &rg);
            if (!gate_off) { ar[s] += cr; ai[s] += ci; }
            if constexpr (DBG) {
                const int64_t j = first + s * kSplitThreads + threadIdx.x;
                dbg_phase[j] = ph;
                dbg_temit[j] = te;
                dbg_delay[j] = rg * b.inv_c;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int64_t j = first + s * kSplitThreads + threadIdx.x;
        if (live[s]) out[j] = band_epilogue(b, ar[s], ai[s], b.i0 + j);
    }
}

int64_t split_tiles(int64_t i0, int64_t n) { return n > 0 ? (i0 + n - 1) / kSplitTile - i0 / kSplitTile + 1 : 0; }

}  // namespace

size_t split_recs_bytes(int64_t i0, int64_t n, int32_t n_active) {
    return sizeof(AnchorRec) * (size_t)split_tiles(i0, n) * (size_t)n_active;
}

cudaError_t launch_band_split(const DevBand &b, const DevTx *d_tx, const int32_t *d_active, int32_t n_active,
                              void *d_recs, float2 *d_out, double *dbg_phase, double *dbg_temit, double *dbg_delay,
                              cudaStream_t s) {
    if (b.n <= 0) return cudaSuccess;
    const int64_t t0 = b.i0 / kSplitTile;
    const int64_t n_tiles = split_tiles(b.i0, b.n);
    const int64_t na = n_tiles * n_active;
    AnchorRec *recs = (AnchorRec *)d_recs;
    if (na > 0) {
        k_split_anchor<<<(unsigned)((na + 127) / 128), 128, 0, s>>>(b, d_tx, d_active, n_active, t0, n_tiles, recs);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const size_t smem = (sizeof(DevTx) + sizeof(AnchorRec)) * (size_t)n_active;
    auto kern = dbg_phase ? k_band_split<true> : k_band_split<false>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<(unsigned)n_tiles, kSplitThreads, smem, s>>>(b, d_tx, d_active, n_active, t0, recs, d_out, dbg_phase,
                                                        dbg_temit, dbg_delay);
    return cudaGetLastError();
}

}  // namespace lpk
