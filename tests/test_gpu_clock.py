"""The receiver clock walk generated on the GPU (LPK_CLOCK_DEVICE_WALK).

The reference draws the white-FM walk sequentially from a xoshiro stream
(src/clock/mod.rs:299-307); the device walk is counter-based, so it is
checked the way the reference checks its own walk: by its statistics
(src/clock/mod.rs:394-422, Allan deviation within 40 %), its deterministic
part (:375-392), chunk invariance (:446-473) and two-band coherence
(:475-510) — plus the fan-out output under it being chunk-invariant.

The flicker part (Flicker, src/clock/mod.rs:55-149) enters the device
clocks as the host stream's own coarse track (lpk_clock_flicker_table),
interpolated on the device: Δt equals the host stream bit for bit where the
clock has no white-FM walk, and a flicker scene rendered with the device
clock matches the oracle, whose clock is the host stream."""
import ctypes as C
import math

import numpy as np
import pytest

from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from lipika_b200 import scene_abi as A
from oracle import oracle as O
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


def _flicker(spec, seed, duration_s):
    n = N.lib().lpk_clock_flicker_len(duration_s)
    tab = np.zeros(n)
    N.check(N.lib().lpk_clock_flicker_table(C.byref(spec), seed, N.dptr(tab), n))
    return tab


def test_flicker_on_device_equals_host_stream(ctx):
    """Deterministic clock + flicker track on the device: Δt equal to the host
    stream (ClockStream::delta_t_at with a flicker floor) bit for bit, in
    chunks at arbitrary offsets."""
    fs, seed = 2.048e6, 77
    spec = A.ClockCfg(0.0, 4e-10, 0.3e-6, 2e-8)
    tab = _flicker(spec, seed, 3.0)
    d = N.BandDesc(fs_hz=fs, lo_hz=1e9, clock_mode=N.LPK_CLOCK_DETERMINISTIC, clock_y0=0.3e-6,
                   clock_offset_s=2e-8, clock_master_rate_hz=fs, clock_seed=seed,
                   flicker_delta_s=tab.ctypes.data_as(C.POINTER(C.c_double)), flicker_n=len(tab))
    L = N.lib()
    h = C.c_void_p()
    N.check(L.lpk_clock_new(C.byref(spec), 0.0, fs, seed, C.byref(h)))
    n = 6_000_000
    t = np.arange(n, dtype=np.float64) / fs
    host = np.zeros(n)
    N.check(L.lpk_clock_delta_t(h, N.dptr(t), n, N.dptr(host)))
    L.lpk_clock_free(h)
    dev = np.concatenate([_delta(ctx, d, i0, min(1_234_567, n - i0)) for i0 in range(0, n, 1_234_567)])
    assert dev.tobytes() == host.tobytes()
    assert np.std(host - (2e-8 + 0.3e-6 * t)) > 0.0  # the flicker is there
    d.flicker_n = 100  # a track shorter than the chunk is refused
    out = np.zeros(10)
    assert L.lpk_clock_device_delta(ctx.h, C.byref(d), n - 10, 10, N.dptr(out)) == N.LPK_EINVAL


def test_flicker_adds_to_the_device_walk(ctx):
    """Walk + flicker: the device Δt minus the same walk without the track
    is the interpolated flicker (up to the rounding of the sums)."""
    fs, seed = 1e6, 5
    spec = A.ClockCfg(1e-11, 1e-10, 0.0, 0.0)
    tab = _flicker(spec, seed, 2.0)
    d = _desc(fs, 1e-11, seed=seed)
    plain = _delta(ctx, d, 500_000, 1_000_000)
    d.flicker_delta_s = tab.ctypes.data_as(C.POINTER(C.c_double))
    d.flicker_n = len(tab)
    both = _delta(ctx, d, 500_000, 1_000_000)
    x = (np.arange(500_000, 1_500_000) / fs) * 128.0
    m = np.floor(x).astype(np.int64)
    fr = x - np.floor(x)
    fl = tab[m] * (1.0 - fr) + tab[m + 1] * fr
    assert np.max(np.abs((both - plain) - fl)) <= 4 * np.spacing(np.max(np.abs(both)))


@pytest.mark.parametrize("batched", [False, True])
def test_flicker_scene_matches_oracle(ctx, batched):
    """A dual-band receiver whose clock has a flicker floor and no white-FM
    walk (so the host stream is deterministic given its seed), 0.3 s, noise
    off: the device clock's render (per band with the FP64 kernel, or the
    batched split path) against the oracle, whose clock is the host stream,
    within 1e-5 of max|oracle| per band; both bands share one flicker
    track."""
    clock = cfg.Clock(allan_deviation_1s=0.0, flicker_floor=5e-10, frequency_offset_y0=0.5e-6,
                      initial_time_offset_s=1e-7)
    sc = scenes.config_c1(duration_s=0.3, clock=clock, noise=False)
    prep = P.Prepared(sc, ctx)
    parts: dict = {}
    if batched:
        prep.generate_scene(2026, 0.1, lambda w, c: parts.setdefault(w, []).append(c) and False, noise=False,
                            device_clock=True, split=True)
    else:
        for w, (r, b) in enumerate(prep.work()):
            prep.generate_band(r, b, 2026, w, 100_003, lambda c, w=w: parts.setdefault(w, []).append(c) and False,
                               noise=False, device_clock=True)
    osc = O.Scene(sc)
    for w, (r, b) in enumerate(prep.work()):
        got = np.concatenate(parts[w]).astype(np.complex128)
        ref = osc.generate_band(r, b, 2026, w, 1 << 20, 4, O.NOISE_NONE)["iq"]
        assert got.shape == ref.shape
        err = float(np.max(np.abs(got - ref))) / float(np.max(np.abs(ref)))
        assert err <= 1e-5, (w, err)
    prep.close()
