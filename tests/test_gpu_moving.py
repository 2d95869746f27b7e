"""A receiver on a circular Keplerian orbit (LPK_RX_KEPLER).

The reference positions such a receiver per sample at the rounded absolute
UTC time (receiver.trajectory.position_ecef_batch(epoch + t_utc),
src/pipeline.rs:929-931; CircularKeplerian::position_ecef,
src/geometry/kepler.rs:32-85). Here the device evaluates the same orbit
expression per sample on the exact paths; the split path fits the receiver's
motion into each tile's anchors and restores the rounding of the receiver's
query per sample, like the transmitter queries. Checked on the dual-band
scene with its receiver put on a 6,900 km orbit, noise off:

* the all-FP64 kernel (per band) and the batched split path against the
  oracle (whose receiver positions come from the host's libm), IQ within
  1e-5 of max|oracle| per band;
* every fast-path (sample, transmitter) of the split path against the
  reference-exact solve in the same kernel: delay <= 1 ps, carrier phase
  <= 1e-6 rad, and split vs all-FP64 IQ <= 1e-5;
* the split path byte-identical across chunkings.
"""
import numpy as np
import pytest

from lipika_b200 import accuracy
from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from lipika_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

IQ_RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _moving_scene(duration_s, clock=None):
    sc = W.config_c1(duration_s=duration_s, noise=False,
                     clock=clock or cfg.Clock(frequency_offset_y0=0.4e-6, initial_time_offset_s=2e-8))
    sc.receivers[0].trajectory = W._kepler(6_900_000.0, 60.0, 30.0, 100.0)
    return sc


def _rel(got, ref):
    ref = ref.astype(np.complex128)
    return float(np.max(np.abs(got.astype(np.complex128) - ref))) / float(np.max(np.abs(ref)))


def test_descriptor_is_the_orbit(ctx):
    prep = P.Prepared(_moving_scene(0.1), ctx)
    for w, (r, b) in enumerate(prep.work()):
        d = prep.band_desc(r, b, 2026, w)
        assert d.rx_kind == N.LPK_RX_KEPLER
        assert d.rx_orbit.semi_major_axis_m == 6_900_000.0 and d.rx_orbit.epoch_unix == W.EPOCH
    prep.close()


@pytest.mark.parametrize("path", ["fp64_per_band", "split_batched"])
def test_moving_receiver_matches_oracle(ctx, path):
    sc = _moving_scene(0.25)
    prep = P.Prepared(sc, ctx)
    parts: dict = {}
    if path == "split_batched":
        prep.generate_scene(2026, 0.1, lambda w, c: parts.setdefault(w, []).append(c) and False, noise=False,
                            device_clock=True, split=True)
    else:
        for w, (r, b) in enumerate(prep.work()):
            prep.generate_band(r, b, 2026, w, 100_003, lambda c, w=w: parts.setdefault(w, []).append(c) and False,
                               noise=False)
    osc = O.Scene(sc)
    for w, (r, b) in enumerate(prep.work()):
        got = np.concatenate(parts[w])
        ref = osc.generate_band(r, b, 2026, w, 1 << 20, 4, O.NOISE_NONE)["iq"]
        assert got.shape == ref.shape
        assert _rel(got, ref) <= IQ_RTOL, (w, _rel(got, ref))
    prep.close()


def test_moving_receiver_split_accuracy(ctx):
    """Whole 2 s scene: the split path's delay and carrier phase per
    fast-path (sample, transmitter) against the reference-exact FP64 solve
    with the receiver at its rounded query time, and split vs all-FP64 IQ."""
    prep = P.Prepared(_moving_scene(2.0), ctx)
    res = accuracy.scene_accuracy(ctx, prep)
    prep.close()
    print(res)
    assert res["txrx_fast"] > 0.99 * (res["txrx_fast"] + res["txrx_exact"])
    assert res["delay_ps"] <= 1.0
    assert res["phase_rad"] <= 1e-6
    assert res["iq_rel"] <= IQ_RTOL


def test_moving_receiver_split_chunk_invariant(ctx):
    prep = P.Prepared(_moving_scene(0.3), ctx)
    r, b = prep.work()[1]  # the 2.048 MS/s band, six C/A transmitters
    outs = []
    for chunk in (1 << 20, 77_777):
        parts = []
        prep.generate_band(r, b, 2026, 1, chunk, lambda c: parts.append(c) and False, noise=False,
                           device_clock=True, split=True)
        outs.append(np.concatenate(parts))
    assert outs[0].tobytes() == outs[1].tobytes()
    prep.close()



def test_mixed_batch_stationary_and_orbiting_receivers(ctx):
    """One batch holding a stationary and an orbiting receiver (the batch then
    runs its orbit-capable kernels, which take the stationary receiver's
    tiles down the stationary code): every unit within 1e-5 of the oracle,
    and the stationary receiver's output equal bit for bit to the same
    receiver batched alone."""
    import copy
    sc = W.config_c1(duration_s=0.2, noise=False,
                     clock=cfg.Clock(frequency_offset_y0=0.4e-6, initial_time_offset_s=2e-8))
    moving = copy.deepcopy(sc.receivers[0])
    moving.name = "leo_rx"
    moving.trajectory = W._kepler(6_900_000.0, 60.0, 30.0, 100.0)
    sc.receivers.append(moving)
    prep = P.Prepared(sc, ctx)
    parts: dict = {}
    prep.generate_scene(2026, 0.1, lambda w, c: parts.setdefault(w, []).append(c) and False, noise=False,
                        device_clock=True, split=True)
    osc = O.Scene(sc)
    kinds = set()
    for w, (r, b) in enumerate(prep.work()):
        kinds.add(prep.band_desc(r, b, 2026, w).rx_kind)
        got = np.concatenate(parts[w])
        ref = osc.generate_band(r, b, 2026, w, 1 << 20, 4, O.NOISE_NONE)["iq"]
        assert _rel(got, ref) <= IQ_RTOL, (w, _rel(got, ref))
    assert kinds == {N.LPK_RX_STATIONARY, N.LPK_RX_KEPLER}
    prep.close()
    alone = W.config_c1(duration_s=0.2, noise=False,
                        clock=cfg.Clock(frequency_offset_y0=0.4e-6, initial_time_offset_s=2e-8))
    p2 = P.Prepared(alone, ctx)
    solo: dict = {}
    p2.generate_scene(2026, 0.1, lambda w, c: solo.setdefault(w, []).append(c) and False, noise=False,
                      device_clock=True, split=True)
    for w in solo:  # the stationary receiver's units come first in both scenes
        assert np.concatenate(solo[w]).tobytes() == np.concatenate(parts[w]).tobytes()
    p2.close()
