"""The split-precision fan-out (LPK_SOLVER_SPLIT) against the all-FP64
reference-semantics kernel and the CPU oracle.

Bars (the target of the split path):
  * emission delay within 1 ps of the FP64 reference solve;
  * carrier phase within 1e-6 rad of the FP64 reference phase;
  * chip / bit / symbol indices bit-exact (a flipped index flips or zeroes a
    contribution, far outside the IQ tolerance below);
  * IQ within 1e-5 x max|reference|.
"""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from oracle import oracle as O
from tests import scenes

pytestmark = pytest.mark.gpu

DELAY_TOL_S = 1e-12
PHASE_TOL_RAD = 1e-6
IQ_RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _contrib(ctx, d, tx, i0, n, solver):
    d.solver = solver
    out = (N.CF32 * n)()
    ph, te, rg = np.zeros(n), np.zeros(n), np.zeros(n)
    N.check(N.lib().lpk_tx_contribution(ctx.h, C.byref(d), tx, i0, n, None, None, out, N.dptr(ph), N.dptr(te),
                                        N.dptr(rg)), ctx.h)
    iq = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_float)), (2 * n,)).view(np.complex64).copy()
    return iq, ph, te, rg / 299792458.0


def _check_split_vs_reference(ctx, scene, starts, n, clock_mode=N.LPK_CLOCK_DEVICE_WALK):
    prep = P.Prepared(scene, ctx)
    worst = {"delay": 0.0, "phase": 0.0, "iq": 0.0}
    for (r, b) in prep.work():
        d = prep.band_desc(r, b, 2026, 0)
        d.clock_mode = clock_mode
        for tx in prep.active(r, b):
            for i0 in starts:
                i0 = min(i0, max(prep.n_samples(r, b) - n, 0))
                ref = _contrib(ctx, d, tx, i0, n, N.LPK_SOLVER_REFERENCE)
                spl = _contrib(ctx, d, tx, i0, n, N.LPK_SOLVER_SPLIT)
                dd = float(np.max(np.abs(spl[3] - ref[3])))
                dp = float(np.max(np.abs(np.angle(np.exp(1j * (spl[1] - ref[1]))))))
                scale = float(np.max(np.abs(ref[0])))
                di = float(np.max(np.abs(spl[0].astype(np.complex128) - ref[0]))) / max(scale, 1e-30)
                assert dd <= DELAY_TOL_S, (r, b, tx, i0, dd)
                assert dp <= PHASE_TOL_RAD, (r, b, tx, i0, dp)
                assert di <= IQ_RTOL, (r, b, tx, i0, di)
                worst = {k: max(worst[k], v) for k, v in (("delay", dd), ("phase", dp), ("iq", di))}
    prep.close()
    return worst


def test_split_matches_reference_dual_band(ctx):
    w = _check_split_vs_reference(ctx, scenes.config_c1(duration_s=120.0),
                                  starts=[0, 1_234_567, 100_000_000, 245_000_000], n=300_000)
    print("split vs FP64 reference, dual-band scene:", w)


def test_split_matches_reference_every_signal_kind(ctx):
    sc = scenes.config_c4(duration_s=60.0, n_rx=2)
    w = _check_split_vs_reference(ctx, sc, starts=[0, 60_000_000, 122_000_000], n=65_536)
    print("split vs FP64 reference, 64-transmitter scene:", w)


def test_split_handles_anchored_gated_and_deterministic_clock(ctx):
    sc = scenes.config_c4(duration_s=2.0, n_rx=1)
    for t in sc.transmitters:
        if t.kind == "ca_code":
            t.params["nav"] = "off"
        t.signal_epoch_unix = 1_000_000_007.25
    from lipika_b200 import config as cfg
    sc.transmitters[0].gate = cfg.Gate(0.01, [(0.0, 0.003), (0.005, 0.002)], 3.0)
    sc.transmitters[20].gate = cfg.Gate(0.007, [(0.001, 0.004)], 0.0)
    _check_split_vs_reference(ctx, sc, starts=[0, 1_000_000], n=50_000, clock_mode=N.LPK_CLOCK_DETERMINISTIC)


def test_split_band_output_matches_oracle(ctx):
    sc = scenes.config_c1(duration_s=0.1)
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    for w, (r, b) in enumerate(prep.work()):
        parts = []
        prep.generate_band(r, b, 7, w, 1 << 16, lambda c: parts.append(c) and False, noise=False, split=True)
        g = np.concatenate(parts)
        ref = osc.generate_band(r, b, 7, w, 1 << 16, 1, O.NOISE_NONE)["iq"]
        scale = float(np.max(np.abs(ref)))
        assert float(np.max(np.abs(g.astype(np.complex128) - ref))) <= IQ_RTOL * scale
    prep.close()


def test_split_chunk_invariant(ctx):
    sc = scenes.config_c1(duration_s=0.2)
    prep = P.Prepared(sc, ctx)
    outs = []
    for chunk in (1 << 20, 3333):
        got = []
        for w, (r, b) in enumerate(prep.work()):
            parts = []
            prep.generate_band(r, b, 5, w, chunk, lambda c: parts.append(c) and False, noise=True,
                               device_clock=True, split=True)
            got.append(np.concatenate(parts))
        outs.append(got)
    for a, b in zip(*outs):
        assert a.tobytes() == b.tobytes()
    prep.close()


def test_split_with_antenna_matches_reference(ctx):
    """Antenna gain folded into the tiles' amplitude; tiles at a pattern
    discontinuity (0 deg, the cutoff) exact; occlusion flags equal. A
    64-transmitter sky over 300 s at 48 kS/s: transmitters rise and set
    through the cutoff."""
    from lipika_b200 import config as cfg
    sc = scenes.config_c4(duration_s=300.0, n_rx=1, noise=False)
    for b in sc.receivers[0].bands:
        b.sample_rate_hz = 48_000.0
        b.frontend = cfg.Frontend(antenna={"peak_dbi": 3.9, "horizon_dbi": -3.0, "fb_db": 8.5, "cutoff_deg": 10.0})
    prep = P.Prepared(sc, ctx)
    L = N.lib()
    (r, b), = prep.work()
    d = prep.band_desc(r, b, 2026, 0)
    d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
    n = prep.n_samples(r, b)
    act = np.ascontiguousarray(np.asarray(prep.active(r, b), np.int32))
    res = {}
    for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_SPLIT):
        d.solver = solver
        out = np.zeros(n, np.complex64)
        flags = np.zeros(max(act.size, 1), np.uint8)
        ctx.check(L.lpk_band_chunk(ctx.h, C.byref(d), act.ctypes.data_as(N._I32), act.size, 0, n, None, None,
                                   out.ctypes.data_as(N._CF), flags.ctypes.data_as(N._U8)))
        res[solver] = (out, flags[:act.size].copy())
    ref, spl = res[N.LPK_SOLVER_REFERENCE], res[N.LPK_SOLVER_SPLIT]
    scale = float(np.max(np.abs(ref[0])))
    err = float(np.max(np.abs(spl[0].astype(np.complex128) - ref[0]))) / scale
    print(f"split vs FP64 with antenna: IQ {err:.2e} of max; {int(ref[1].sum())} of {act.size} transmitters "
          "above the cutoff at some sample")
    assert 0 < ref[1].sum() < act.size  # some visible, some occluded throughout
    assert err <= IQ_RTOL
    assert np.array_equal(ref[1], spl[1])
    prep.close()


@pytest.mark.parametrize("fs", [2.048e6, 48e3, 4.096e6, 250e3, 8.184e6, 1e6 / 3, 44100.0, 2.5e6 + 0.1,
                                12345.678, 61.44e6])
def test_split_sample_times_are_the_ieee_quotient(ctx, fs):
    """The split fan-out forms t = i / fs with a reciprocal and one fma
    correction (Markstein); every value must be the correctly rounded
    quotient the reference computes (src/pipeline.rs:918), checked against
    numpy's IEEE division over whole bands and far index ranges."""
    L = N.lib()
    n = 1 << 22
    for i0 in (0, n, 1 << 28, (1 << 31) - 17, 10 ** 12 + 3, (1 << 52) - n):
        t = np.zeros(n)
        ctx.check(L.lpk_sample_times(ctx.h, fs, i0, n, t.ctypes.data_as(N._D)))
        ref = np.arange(i0, i0 + n, dtype=np.int64).astype(np.float64) / fs
        bad = np.flatnonzero(t != ref)
        assert bad.size == 0, (fs, i0, bad[:5], t[bad[:5]], ref[bad[:5]])
