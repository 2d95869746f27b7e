"""GPU parity: the sm_100a fan-out against the CPU oracle.

Tolerances (the contract of this backend):
  * emission times, ranges, chip / bit / symbol indices: bit-exact;
  * IQ: |gpu - oracle| <= 1e-5 * max|oracle| per band (CUDA's sin/cos may
    differ from glibc's in the last ulp before the f32 cast);
  * ADC codes on identical f32 inputs: bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from lipika_b200 import scene_abi as A
from oracle import oracle as O
from tests import scenes

pytestmark = pytest.mark.gpu

IQ_RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _assert_iq_close(gpu, ref, rtol=IQ_RTOL):
    assert gpu.shape == ref.shape
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    err = float(np.max(np.abs(gpu.astype(np.complex128) - ref.astype(np.complex128)))) if ref.size else 0.0
    assert err <= rtol * max(scale, 1e-30), f"max err {err:.3e} vs scale {scale:.3e}"


def _gpu_band(prep, r, b, seed, work_idx, chunk, noise):
    chunks = []
    res = prep.generate_band(r, b, seed, work_idx, chunk, lambda c: chunks.append(c) and False, noise)
    return (np.concatenate(chunks) if chunks else np.zeros(0, np.complex64)), res


def _compare_scene(ctx, scene, seed=7, chunk=1 << 16, noise=False, limit=None,
                   time_base=A.LPK_TIME_BASE_SCENE):
    prep = P.Prepared(scene, ctx, time_base, 0.0)
    osc = O.Scene(scene, time_base, 0.0)
    for w, (r, b) in enumerate(prep.work()):
        g, res = _gpu_band(prep, r, b, seed, w, chunk, noise)
        ref = osc.generate_band(r, b, seed, w, chunk, 1, O.NOISE_COUNTER if noise else O.NOISE_NONE)
        _assert_iq_close(g, ref["iq"])
        na = len(osc.active(r, b))
        assert [bool(res.unoccluded[k]) for k in range(na)] == ref["unoccluded"]
    prep.close()


def test_emission_solve_bit_exact(ctx):
    sc = scenes.config_c1(duration_s=2.0)
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    rx = np.array(O.geodetic_to_ecef(55.86, -4.25, 10.0))
    n = 200_000
    t = np.linspace(-0.4, 2.3, n)
    obs = np.ascontiguousarray(np.repeat(rx[:, None], n, axis=1))
    for tx in range(len(sc.transmitters)):
        for iters in (1, 2, 4):
            te, rg = np.zeros(n), np.zeros(n)
            N.check(N.lib().lpk_solve_emission_times(ctx.h, tx, N.dptr(obs), N.dptr(t), n, sc.epoch_unix, iters,
                                                     N.dptr(te), N.dptr(rg)), ctx.h)
            te2, rg2 = np.zeros(n), np.zeros(n)
            O.lib().orc_solve_emission_times(O.lib().orc_scene_traj(osc.h, tx), O.dptr(obs), O.dptr(t), n,
                                             sc.epoch_unix, iters, O.dptr(te2), O.dptr(rg2))
            assert te.tobytes() == te2.tobytes() and rg.tobytes() == rg2.tobytes(), (tx, iters)
    prep.close()


def test_tx_contribution_t_emit_and_range_bit_exact(ctx):
    sc = scenes.config_c4(duration_s=0.2, n_rx=1, noise=False)
    prep = P.Prepared(sc, ctx)
    osc = O.Scene(sc)
    d = prep.band_desc(0, 0, 0, 0)
    d.clock_mode = N.LPK_CLOCK_DETERMINISTIC  # δ = c + y0·t on both sides
    n = 20_000
    i0 = 1_000_003
    for tx in range(0, 64, 5):
        out = (N.CF32 * n)()
        te, rg, ph = np.zeros(n), np.zeros(n), np.zeros(n)
        delta = np.zeros(n)
        N.check(N.lib().lpk_tx_contribution(ctx.h, C.byref(d), tx, i0, n, N.dptr(delta), None, out, N.dptr(ph),
                                            N.dptr(te), N.dptr(rg)), ctx.h)
        t_local = (i0 + np.arange(n)) / d.fs_hz
        dl = d.clock_offset_s + d.clock_y0 * t_local
        tu = t_local - dl
        obs = np.ascontiguousarray(np.repeat(np.array(list(d.rx_ecef))[:, None], n, axis=1))
        te2, rg2 = np.zeros(n), np.zeros(n)
        O.lib().orc_solve_emission_times(O.lib().orc_scene_traj(osc.h, tx), O.dptr(obs), O.dptr(tu), n,
                                         sc.epoch_unix, 2, O.dptr(te2), O.dptr(rg2))
        assert te.tobytes() == te2.tobytes() and rg.tobytes() == rg2.tobytes(), tx
        acc = np.zeros(2 * n, dtype=np.float32)
        O.lib().orc_accumulate(O.fptr(acc), O.lib().orc_scene_signal(osc.h, tx), O.lib().orc_scene_traj(osc.h, tx),
                               O.dptr(obs), O.dptr(t_local), O.dptr(tu), O.dptr(dl), n, d.lo_hz,
                               O.lib().orc_scene_tx_power_w(osc.h, tx), sc.epoch_unix, 2, None)
        g = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_float)), (2 * n,)).view(np.complex64)
        _assert_iq_close(g, acc.view(np.complex64))
    prep.close()


def test_baseband_indices_bit_exact_every_kind(ctx):
    """Chip / bit / symbol values picked by the GPU equal the oracle's for
    every sample: the sign pattern of the contribution of a stationary
    transmitter (constant carrier phase) is the baseband itself."""
    for sig in (scenes.SIG_OOK, scenes.SIG_QAM16):
        sc = scenes.parse(scenes.OOK_QAM_TEMPLATE.replace("@SIGNAL@", sig))
        _compare_scene(ctx, sc, chunk=4096)
    sc = scenes.parse(scenes.BPSK)
    _compare_scene(ctx, sc, chunk=10_000)


def test_small_scenes_match_oracle(ctx):
    for text in (scenes.TWO_TX, scenes.STREAMING, scenes.CW_TWO_CLOCKS):
        _compare_scene(ctx, scenes.parse(text), chunk=8192)


def test_config_c0_prefix_matches_oracle(ctx):
    # one CW GPS transmitter, 2.048 MS/s, walk clock, first 0.25 s.
    _compare_scene(ctx, scenes.config_c0(duration_s=0.25), chunk=1 << 20)


def test_config_c1_prefix_matches_oracle(ctx):
    # BPSK LEO at 48 kS/s + 6 C/A at 2.048 MS/s, walk clock.
    _compare_scene(ctx, scenes.config_c1(duration_s=0.1), chunk=1 << 16)


def test_config_c4_all_kinds_match_oracle(ctx):
    _compare_scene(ctx, scenes.config_c4(duration_s=0.01, n_rx=2), chunk=1 << 14)


def test_anchored_window_and_gate_match_oracle(ctx):
    sc = scenes.config_c4(duration_s=0.02, n_rx=1)
    for t in sc.transmitters:
        if t.kind == "ca_code":
            t.params["nav"] = "off"
    sc.transmitters[0].gate = cfg.Gate(0.01, [(0.0, 0.003), (0.005, 0.002)], 3.0)
    sc.transmitters[20].gate = cfg.Gate(0.007, [(0.001, 0.004)], 0.0)
    _compare_scene(ctx, sc, chunk=8192, time_base=A.LPK_TIME_BASE_ABSOLUTE)


def test_antenna_occlusion_and_frontend_match_oracle(ctx):
    sc = scenes.config_c1(duration_s=0.05)
    for b in sc.receivers[0].bands:
        b.frontend = cfg.Frontend(antenna={"peak_dbi": 3.9, "horizon_dbi": -3.0, "fb_db": 8.5, "cutoff_deg": 5.0},
                                  gain_db=150.0, iip3_dbm=40.0)
    _compare_scene(ctx, sc, chunk=1 << 15)


def test_noise_matches_counter_spec_and_kTB(ctx):
    sc = scenes.parse(scenes.NO_TX)
    prep = P.Prepared(sc, ctx)
    g, _ = _gpu_band(prep, 0, 0, 12345, 0, 1 << 17, True)
    osc = O.Scene(sc)
    ref = osc.generate_band(0, 0, 12345, 0, 1 << 17, 1, O.NOISE_COUNTER)["iq"]
    _assert_iq_close(g, ref, rtol=2e-6)
    p = float(np.mean(np.abs(g.astype(np.complex128)) ** 2))
    assert abs(p / 1e-15 - 1) < 0.02  # tests/multi_transmitter_summation.rs:185
    re, im = g.real.astype(np.float64), g.imag.astype(np.float64)
    assert abs(np.mean(re)) < 5e-4 * np.std(re) * 10
    assert abs(np.corrcoef(re[:-1], re[1:])[0, 1]) < 0.01
    assert abs(np.corrcoef(re, im)[0, 1]) < 0.01
    prep.close()


def test_superposition_one_noise_draw_on_gpu(ctx):  # tests/multi_transmitter_summation.rs:189-242
    both = scenes.parse(scenes.TWO_TX)
    alpha, beta = both.clone(), both.clone()
    alpha.transmitters = [t for t in alpha.transmitters if t.name == "alpha"]
    beta.transmitters = [t for t in beta.transmitters if t.name == "beta"]
    run = lambda s: P.run_scene(s, 99, ctx)[0].iq
    a, b, ab, n = run(alpha), run(beta), run(both), run(scenes.parse(scenes.NO_TX))
    assert float(np.max(np.abs(ab - (a + b - n)))) < 1e-10


def test_chunk_size_invariance_byte_identical(ctx, tmp_path):  # tests/streaming_chunk_invariance.rs
    sc = scenes.parse(scenes.STREAMING)
    P.run_scene_to_dir(sc, 4242, str(tmp_path / "one"), chunk_samples=1 << 22, ctx=ctx)
    P.run_scene_to_dir(sc, 4242, str(tmp_path / "many"), chunk_samples=4096, ctx=ctx)
    mem = P.run_scene(sc, 4242, ctx)
    for out in mem:
        a = (tmp_path / "one" / f"{out.name}.iq.c64").read_bytes()
        b = (tmp_path / "many" / f"{out.name}.iq.c64").read_bytes()
        assert a == b and len(a) == 8 * len(out.iq) > 0
        assert out.iq.astype(np.complex64).tobytes() == a
        side = (tmp_path / "one" / f"{out.name}.iq.json").read_text()
        assert '"n_samples"' in side and "raw complex64" in side


def test_adc_codes_bit_exact_on_identical_inputs(ctx):
    rng = np.random.default_rng(3)
    n = 100_000
    x = (rng.standard_normal(2 * n) * 0.6).astype(np.float32)
    x[:8] = [0.5, -0.5, 2.0, -3.0, 1 / 14, -1 / 14, 0.0, -0.0]
    for bits, fs, gain in ((4, 1.0, None), (8, 0.8, 6.0), (12, 2.5, -3.0)):
        fe = A.FrontendCfg(has_adc=1, adc_bits=bits, adc_full_scale_v=fs, has_gain=int(gain is not None),
                           gain_db=gain or 0.0)
        ch = O.RxChain()
        O.lib().orc_rx_chain_from_config(C.byref(fe), 1, C.byref(ch))
        ref = x.copy()
        O.lib().orc_rx_apply_post_sum(C.byref(ch), O.fptr(ref), n)
        d = N.BandDesc(fs_hz=1.0)
        k = 0
        if gain is not None:
            d.post[k] = N.PostOp(N.LPK_POST_GAIN, 0, gain)
            k += 1
        d.post[k] = N.PostOp(N.LPK_POST_ADC, bits, fs)
        d.n_post = k + 1
        g = x.copy()
        N.check(N.lib().lpk_rx_chain_apply(ctx.h, C.byref(d), g.ctypes.data_as(C.POINTER(N.CF32)), n), ctx.h)
        assert g.tobytes() == ref.tobytes(), bits


def test_render_window_stops_and_reports(ctx):
    sky = cfg.Sky(scenes.config_c4(duration_s=1.0, n_rx=1).transmitters[:16])
    rx = cfg.Receiver("g", cfg.Trajectory("stationary_geodetic", {"lat_deg": 55.86, "lon_deg": -4.25, "h_m": 10.0}))
    band = cfg.Band("l1", 1575.42e6, 1.0e6, 290.0, 0.0)
    seen = []

    def sink(c):
        seen.append(len(c))
        return len(seen) == 3

    s = P.render_window(sky, rx, band, scenes.EPOCH, 0.5, P.WindowOptions(seed=1, chunk_samples=50_000), sink, ctx)
    assert s.stopped_early and s.n_samples_emitted == 150_000 and s.n_samples_window == 500_000
    assert len(s.contributing_transmitters) > 0


def test_errors_are_status_codes_not_crashes(ctx):
    d = N.BandDesc(fs_hz=-1.0)
    out = (N.CF32 * 4)()
    act = (C.c_int32 * 1)(0)
    assert N.lib().lpk_band_chunk(ctx.h, C.byref(d), act, 1, 0, 4, None, None, out, None) == N.LPK_EINVAL
    d = N.BandDesc(fs_hz=1e6, clock_mode=N.LPK_CLOCK_DETERMINISTIC)
    act = (C.c_int32 * 1)(99999)
    assert N.lib().lpk_band_chunk(ctx.h, C.byref(d), act, 1, 0, 4, None, None, out, None) == N.LPK_EINVAL
    assert b"out of range" in N.lib().lpk_last_error(ctx.h)
