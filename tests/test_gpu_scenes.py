"""Parity on every BASELINE scene, at full size and against the CPU oracle.

* Whole scenes (dual-band 120 s, 24 C/A x 32 receivers 30 s, the 600 s long
  coherent scene with L1 at 8.184 MS/s, 64 transmitters x 16 receivers 60 s):
  every band sample rendered by the split-precision fan-out and by the
  all-FP64 kernel (noise off, clock walk on the device). For every
  fast-path (sample, transmitter) the split kernel's emission delay and
  carrier phase are compared with the reference-exact FP64 solve in the
  same kernel (lpk_split_accuracy); the two renders are compared per band.
  Bars: delay <= 1 ps, carrier phase <= 1e-6 rad, IQ <= 1e-5 x max|IQ|.
* Windows against the oracle (the CPU restatement of the reference loop):
  a late second of the 600 s scene (590-591 s), a prefix of the 24 x 32
  scene covering every rate class, and 0.2 s of the 64 x 16 scene. IQ within
  1e-5 x max|oracle| per band; the FP64 kernel's emission times bit-exact at
  the late window.
"""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import accuracy
from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from lipika_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DELAY_TOL_PS = 1.0
PHASE_TOL_RAD = 1e-6
IQ_RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _oracle_threads():
    import os
    return max(1, os.cpu_count() or 1)


@pytest.mark.parametrize("name", ["c1", "c2", "c3", "c4"])
def test_whole_scene_accuracy(ctx, name):
    sc = {"c1": lambda: W.config_c1(noise=False), "c2": lambda: W.config_c2(noise=False),
          "c3": lambda: W.config_c3(noise=False), "c4": lambda: W.config_c4(noise=False)}[name]()
    prep = P.Prepared(sc, ctx)
    acc = accuracy.scene_accuracy(ctx, prep)
    prep.close()
    print(f"{name}: {acc}")
    assert acc["txrx_fast"] > 0
    assert acc["delay_ps"] <= DELAY_TOL_PS, acc
    assert acc["phase_rad"] <= PHASE_TOL_RAD, acc
    assert acc["iq_rel"] <= IQ_RTOL, acc


def _band_chunk(ctx, d, act, i0, n):
    out = np.zeros(n, np.complex64)
    a = np.ascontiguousarray(np.asarray(act, np.int32))
    ctx.check(N.lib().lpk_band_chunk(ctx.h, C.byref(d), a.ctypes.data_as(N._I32), a.size, i0, n, None, None,
                                     out.ctypes.data_as(N._CF), None))
    return out


def test_long_scene_late_window_matches_oracle(ctx):
    """590-591 s of the 600 s scene (L1 at 8.184 MS/s): the split and FP64
    kernels against the oracle's render of the same window, and the FP64
    kernel's emission times bit-exact against the oracle's solve."""
    clock = cfg.Clock(frequency_offset_y0=0.5e-6, initial_time_offset_s=2e-7)  # deterministic: same Δt
    sc = W.config_c3(clock=clock, noise=False)
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    for w, (r, b) in enumerate(prep.work()):
        fs = sc.receivers[r].bands[b].sample_rate_hz
        i0, n = int(590 * fs), int(fs)
        act = prep.active(r, b)
        ref = osc.generate_window(r, b, 2026, w, i0, n, 1 << 20, _oracle_threads(), O.NOISE_NONE)
        scale = float(np.max(np.abs(ref)))
        d = prep.band_desc(r, b, 2026, w)
        d.clock_mode = N.LPK_CLOCK_DETERMINISTIC
        d.noise_power_w = 0.0
        for solver in (N.LPK_SOLVER_SPLIT, N.LPK_SOLVER_REFERENCE):
            d.solver = solver
            got = _band_chunk(ctx, d, act, i0, n)
            if scale == 0.0:  # the one-shot BPSK frame ended at 30 s: silence
                assert not np.any(got)
                continue
            err = float(np.max(np.abs(got.astype(np.complex128) - ref))) / scale
            print(f"unit {w} solver {solver}: {err:.2e} of max|oracle| over {n} samples at 590 s")
            assert err <= IQ_RTOL
    # emission times of the FP64 kernel at the late window, bit-exact
    L = N.lib()
    rx = np.array(prep.band_desc(0, 1, 2026, 1).rx_ecef[:])
    fs = 8.184e6
    i = np.arange(int(590.5 * fs), int(590.5 * fs) + 200_000, dtype=np.int64)
    tl = i.astype(np.float64) / fs
    tu = tl - (0.0 + (2e-7 + 0.5e-6 * tl))
    obs = np.ascontiguousarray(np.repeat(rx[:, None], len(tu), axis=1))
    for tx in prep.active(0, 1):
        te_g, rg_g = np.zeros(len(tu)), np.zeros(len(tu))
        ctx.check(L.lpk_solve_emission_times(ctx.h, tx, N.dptr(obs), N.dptr(tu), len(tu), sc.epoch_unix, 2,
                                             N.dptr(te_g), N.dptr(rg_g)))
        te_o, rg_o = np.zeros(len(tu)), np.zeros(len(tu))
        O.lib().orc_solve_emission_times(O.lib().orc_scene_traj(osc.h, tx), O.dptr(obs), O.dptr(tu), len(tu),
                                         sc.epoch_unix, 2, O.dptr(te_o), O.dptr(rg_o))
        assert np.array_equal(te_g, te_o) and np.array_equal(rg_g, rg_o), tx
    prep.close()


def test_batched_scene_prefix_matches_oracle(ctx):
    """The 24 C/A x 32 receiver scene (1-3 bands per receiver at 48 k -
    4.096 MS/s) through the batched split path, against the oracle per
    unit: the first 50 ms of every work unit, every rate class present."""
    sc = W.config_c2(duration_s=0.05, clock_walk=False, noise=False)
    rates = {b.sample_rate_hz for rx in sc.receivers for b in rx.bands}
    assert rates == {48_000.0, 250_000.0, 2.048e6, 4.096e6}
    prep = P.Prepared(sc, ctx)
    parts: dict = {}
    prep.generate_scene(2026, 0.02, lambda w, c: parts.setdefault(w, []).append(c) and False, noise=False,
                        device_clock=True, split=True)
    osc = O.Scene(sc)
    worst = 0.0
    for w, (r, b) in enumerate(prep.work()):
        got = np.concatenate(parts[w])
        ref = osc.generate_band(r, b, 2026, w, 1 << 20, _oracle_threads(), O.NOISE_NONE)["iq"]
        assert got.shape == ref.shape
        scale = float(np.max(np.abs(ref)))
        err = float(np.max(np.abs(got.astype(np.complex128) - ref))) / scale
        worst = max(worst, err)
        assert err <= IQ_RTOL, (w, err)
    print(f"24 x 32 scene, {len(parts)} units: worst {worst:.2e} of max|oracle|")
    prep.close()


def test_sixty_four_transmitter_window_matches_oracle(ctx):
    """0.2 s of the 64 x 16 scene on every receiver: the split kernel with
    the host clock stream (bit-identical to the oracle's) against the
    oracle's render."""
    sc = W.config_c4(duration_s=0.2, noise=False)
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    worst = 0.0
    for w, (r, b) in enumerate(prep.work()):
        parts = []
        prep.generate_band(r, b, 2026, w, 1 << 18, lambda c: parts.append(c) and False, noise=False, split=True)
        got = np.concatenate(parts)
        ref = osc.generate_band(r, b, 2026, w, 1 << 18, _oracle_threads(), O.NOISE_NONE)["iq"]
        scale = float(np.max(np.abs(ref)))
        err = float(np.max(np.abs(got.astype(np.complex128) - ref))) / scale
        worst = max(worst, err)
        assert err <= IQ_RTOL, (w, err)
    print(f"64 x 16 scene, 0.2 s: worst {worst:.2e} of max|oracle|")
    prep.close()


@pytest.mark.parametrize("name", ["c1", "c4"])
def test_tuned_fp64_kernel_within_tolerance(ctx, name):
    """The tuned all-FP64 fan-out (LPK_SOLVER_FP64_TUNED: lerp by 1/dt,
    phases reduced modulo 2π before one FP64 sincos) against the
    reference-exact FP64 kernel on every band of the scene: IQ within
    1e-5 x max|IQ|."""
    import torch
    sc = {"c1": lambda: W.config_c1(duration_s=8.0, noise=False),
          "c4": lambda: W.config_c4(duration_s=4.0, noise=False)}[name]()
    prep = P.Prepared(sc, ctx)
    L = N.lib()
    worst = 0.0
    for w, (r, b) in enumerate(prep.work()):
        d = prep.band_desc(r, b, 2026, w)
        d.clock_mode = N.LPK_CLOCK_DEVICE_WALK
        n = prep.n_samples(r, b)
        act = (C.c_int32 * max(len(prep.active(r, b)), 1))(*prep.active(r, b))
        outs = []
        for solver in (N.LPK_SOLVER_REFERENCE, N.LPK_SOLVER_FP64_TUNED):
            d.solver = solver
            o = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
            ctx.check(L.lpk_band_chunk_device(ctx.h, C.byref(d), act, len(prep.active(r, b)), 0, n, None, None,
                                              o.data_ptr(), None))
            ctx.check(L.lpk_sync(ctx.h))
            outs.append(o.view(n, 2).double())
        scale = float(torch.linalg.vector_norm(outs[0], dim=1).max())
        err = float(torch.linalg.vector_norm(outs[1] - outs[0], dim=1).max()) / scale
        worst = max(worst, err)
        assert err <= IQ_RTOL, (w, err)
    print(f"{name}: tuned FP64 vs reference FP64, worst {worst:.2e} of max|IQ|")
    prep.close()
