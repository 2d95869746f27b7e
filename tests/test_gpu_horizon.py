"""The horizon gate (src/channel/horizon.rs) on the GPU: with an antenna
cutoff, blocks of samples skip transmitters certainly below it. The gate
must change no output bit (the per-sample path gives those samples zero
gain), and it must actually skip work on a sky where many transmitters are
below the horizon (tests/horizon_gate.rs checks the same two things)."""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from oracle import oracle as O
from tests import scenes

pytestmark = pytest.mark.gpu

ANTENNA = {"peak_dbi": 3.9, "horizon_dbi": -3.0, "fb_db": 8.5, "cutoff_deg": 10.0}


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _sky(duration_s=0.2, n_rx=2):
    sc = scenes.config_c4(duration_s=duration_s, n_rx=n_rx, noise=False)
    for rx in sc.receivers:
        for b in rx.bands:
            b.frontend = cfg.Frontend(antenna=dict(ANTENNA))
    return sc


def _stats(ctx, reset=True):
    t, s = C.c_int64(), C.c_int64()
    ctx.check(N.lib().lpk_gate_stats(ctx.h, C.byref(t), C.byref(s), 1 if reset else 0))
    return t.value, s.value


def test_gate_skips_work_and_matches_oracle(ctx):
    sc = _sky()
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    _stats(ctx)
    for w, (r, b) in enumerate(prep.work()):
        chunks = []
        res = prep.generate_band(r, b, 7, w, 1 << 16, lambda c: chunks.append(c) and False, noise=False)
        g = np.concatenate(chunks)
        ref = osc.generate_band(r, b, 7, w, 1 << 16, 1, O.NOISE_NONE)
        scale = max(float(np.max(np.abs(ref["iq"]))), 1e-30)
        assert float(np.max(np.abs(g.astype(np.complex128) - ref["iq"]))) <= 1e-5 * scale
        na = len(osc.active(r, b))
        assert [bool(res.unoccluded[k]) for k in range(na)] == ref["unoccluded"]
    tested, skipped = _stats(ctx)
    print(f"FP64 path: {skipped} of {tested} (block, transmitter) pairs skipped by the horizon gate")
    assert tested > 0 and 0.2 * tested < skipped < tested
    prep.close()


def test_gate_in_the_batch_changes_no_bit(ctx):
    sc = _sky()
    prep = P.Prepared(sc, ctx)
    units = []
    for w, (r, b) in enumerate(prep.work()):
        d = prep.band_desc(r, b, 7, w)
        d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
        d.solver = N.LPK_SOLVER_SPLIT
        units.append((d, prep.active(r, b), prep.n_samples(r, b)))
    single = []
    for d, act, n in units:
        out = np.zeros(n, np.complex64)
        a = np.ascontiguousarray(np.asarray(act, np.int32))
        ctx.check(N.lib().lpk_band_chunk(ctx.h, C.byref(d), a.ctypes.data_as(N._I32), a.size, 0, n, None, None,
                                         out.ctypes.data_as(N._CF), None))
        single.append(out)
    _stats(ctx)
    got = N.Batch(ctx, units, round_s=0.05).render()
    tested, skipped = _stats(ctx)
    print(f"batch: {skipped} of {tested} (tile, transmitter) pairs skipped")
    assert 0.2 * tested < skipped < tested
    for x, y in zip(got, single):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    prep.close()
