"""The receiver clock walk generated on the GPU (LPK_CLOCK_DEVICE_WALK).

The reference draws the white-FM walk sequentially from a xoshiro stream
(src/clock/mod.rs:299-307); the device walk is counter-based, so it is
checked the way the reference checks its own walk: by its statistics
(src/clock/mod.rs:394-422, Allan deviation within 40 %), its deterministic
part (:375-392), chunk invariance (:446-473) and two-band coherence
(:475-510) — plus the fan-out output under it being chunk-invariant."""
import ctypes as C
import math

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _desc(fs, allan, y0=0.0, c0=0.0, master=None, seed=7):
    d = N.BandDesc(fs_hz=fs, lo_hz=1e9, clock_mode=N.LPK_CLOCK_DEVICE_WALK, clock_allan_1s=allan,
                   clock_y0=y0, clock_offset_s=c0, clock_master_rate_hz=master or fs, clock_seed=seed)
    return d


def _delta(ctx, d, i0, n):
    out = np.zeros(n)
    N.check(N.lib().lpk_clock_device_delta(ctx.h, C.byref(d), i0, n, N.dptr(out)), ctx.h)
    return out


def test_deterministic_part_exact(ctx):
    d = _desc(1e6, 0.0, y0=5e-6)
    out = _delta(ctx, d, 0, 1_000_000)
    t = np.arange(1_000_000) / 1e6
    assert np.array_equal(out, 0.0 + (0.0 + 5e-6 * t))


def test_chunk_invariance_bit_exact(ctx):
    d = _desc(2.048e6, 1e-10, y0=1e-6, c0=3e-8, seed=11)
    whole = _delta(ctx, d, 0, 3_000_000)
    parts = np.concatenate([_delta(ctx, d, i0, min(777_777, 3_000_000 - i0)) for i0 in range(0, 3_000_000, 777_777)])
    assert whole.tobytes() == parts.tobytes()
    other = N.Context(0)  # a fresh context (fresh carry cache) reproduces it too
    again = _delta(other, d, 1_500_000, 1_000)
    other.close()
    assert again.tobytes() == whole[1_500_000:1_501_000].tobytes()


def test_allan_deviation_recovers_target(ctx):  # src/clock/mod.rs:394-422
    fs = 1e6
    d = _desc(fs, 1e-11, seed=7)
    track = np.concatenate([_delta(ctx, d, i0, 5_000_000) for i0 in range(0, 60_000_000, 5_000_000)])
    steps = np.diff(track[::int(fs)])
    assert abs(np.std(steps) / 1e-11 - 1) < 0.4
    inc = np.diff(track[:2_000_000])
    assert abs(np.std(inc) / (1e-11 / math.sqrt(fs)) - 1) < 0.01
    assert abs(np.corrcoef(inc[:-1], inc[1:])[0, 1]) < 0.01
    assert abs(np.mean(inc)) < 5 * np.std(inc) / math.sqrt(len(inc))


def test_two_bands_coherent(ctx):  # src/clock/mod.rs:475-510
    master, low = 2.048e6, 48_000.0
    hi = _delta(ctx, _desc(master, 1e-11, y0=0.3e-6, master=master, seed=99), 0, 30_000)
    lo = _delta(ctx, _desc(low, 1e-11, y0=0.3e-6, master=master, seed=99), 0, 500)
    for j in range(500):
        x = (j / low) * master
        k0 = int(math.floor(x))
        fr = x - k0
        ref = hi[k0] * (1 - fr) + hi[k0 + 1] * fr
        assert abs(lo[j] - ref) <= max(1e-9 * abs(ref), 1e-18)


def test_band_output_chunk_invariant_under_device_clock(ctx):
    sc = scenes.config_c1(duration_s=0.3)
    prep = P.Prepared(sc, ctx)
    outs = []
    for chunk in (1 << 20, 10_007):
        got = []
        for w, (r, b) in enumerate(prep.work()):
            parts = []
            prep.generate_band(r, b, 5, w, chunk, lambda c: parts.append(c) and False, noise=True,
                               device_clock=True)
            got.append(np.concatenate(parts))
        outs.append(got)
    for a, b in zip(*outs):
        assert a.tobytes() == b.tobytes()
    prep.close()
