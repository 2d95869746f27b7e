"""Pin the CPU oracle to the reference's own known-answer tests.

Each test restates an assertion of the reference's test suite (file:line
cited) and runs it against the C oracle, so the oracle is trusted before the
CUDA backend is compared with it.
"""
import ctypes as C
import math

import numpy as np
import pytest

from lipika_b200 import config as cfg
from lipika_b200 import scene_abi as A
from oracle import oracle as O
from tests import scenes

EPOCH = scenes.EPOCH
SPEED_OF_LIGHT = 299792458.0


def _tx(kind, params, carrier=1e9, **kw):
    return cfg.Transmitter(name="t", carrier_hz=carrier, kind=kind, params=params,
                           trajectory=cfg.Trajectory("stationary_ecef", {"x_m": 7e6, "y_m": 0.0, "z_m": 0.0}), **kw)


def _signal(tx, render_epoch=EPOCH, time_base=A.LPK_TIME_BASE_SCENE, default_epoch=0.0):
    sc = O.Scene(cfg.Scene(render_epoch, 1.0, [tx], []), time_base, default_epoch)
    return sc, O.lib().orc_scene_signal(sc.h, 0)


def _eval(sig, t):
    t = np.ascontiguousarray(t, dtype=np.float64)
    out = np.zeros(2 * len(t), dtype=np.float32)
    O.lib().orc_signal_eval(sig, O.dptr(t), len(t), O.fptr(out))
    return out.view(np.complex64)


# ---------------------------------------------------------------- geometry
def test_glasgow_ecef_matches_reference():  # src/geometry/ecef.rs:29-37
    p = O.geodetic_to_ecef(55.86, -4.25, 10.0)
    for got, exp in zip(p, [3577894.5228608, -265883.49155448, 5255718.21468305]):
        assert abs(got / exp - 1) < 1e-9


def test_equator_on_x_axis():  # src/geometry/ecef.rs:40-45
    p = O.geodetic_to_ecef(0.0, 0.0, 0.0)
    assert abs(p[0] / 6378137.0 - 1) < 1e-12 and abs(p[1]) < 1e-6 and abs(p[2]) < 1e-6


def _kep(a=6378137.0 + 20200000.0, inc=55.0, raan=0.0, ta=30.0, ep=1_700_000_000.0):
    return A.TrajectoryCfg(kind=A.LPK_TRAJ_CIRCULAR_KEPLERIAN, semi_major_axis_m=a, inclination_deg=inc,
                           raan_deg=raan, true_anomaly_deg_at_epoch=ta, epoch_unix=ep)


def test_kepler_gps_radius():  # src/geometry/kepler.rs:112-124
    k = _kep(ta=0.0, ep=0.0)
    p = np.zeros(3)
    O.lib().orc_kepler_position_ecef(C.byref(k), 0.0, O.dptr(p))
    assert abs(np.linalg.norm(p) / (6378137.0 + 20200000.0) - 1) < 1e-9


def test_precomputed_matches_underlying_sub_metre():  # src/geometry/precomputed.rs:206-225
    k = _kep()
    tr = O.Traj()
    assert O.lib().orc_traj_sample(C.byref(k), 1_700_000_000.0, 60.0, 0.01, C.byref(tr)) == 0
    for i in range(50):
        t = 1_700_000_000.0 + 60.0 * i / 50
        exact, approx = np.zeros(3), np.zeros(3)
        O.lib().orc_kepler_position_ecef(C.byref(k), t, O.dptr(exact))
        O.lib().orc_traj_position(C.byref(tr), t, O.dptr(approx))
        for ax in range(3):
            assert abs(exact[ax] - approx[ax]) <= max(1e-6 * abs(exact[ax]), 1e-3)
    O.lib().orc_traj_free(C.byref(tr))


def test_path_bounds_cover_queries():  # src/geometry/precomputed.rs:162-201
    k = _kep(a=6928137.0, inc=53.0, raan=10.0, ta=0.0)
    tr = O.Traj()
    O.lib().orc_traj_sample(C.byref(k), 1_700_000_000.0, 30.0, 0.01, C.byref(tr))
    v, r = tr.max_speed_m_s, tr.max_radius_m
    assert 6900.0 < v < 7700.0
    assert abs(r / 6928137.0 - 1) < 1e-9
    prev = None
    for i in range(4000):
        t = 1_700_000_000.0 - 2.0 + i * 0.0087
        p = np.zeros(3)
        O.lib().orc_traj_position(C.byref(tr), t, O.dptr(p))
        assert np.linalg.norm(p) <= r * (1 + 1e-12)
        if prev is not None:
            assert np.linalg.norm(p - prev[1]) <= v * (t - prev[0]) * (1 + 1e-9) + 1e-6
        prev = (t, p)
    O.lib().orc_traj_free(C.byref(tr))


# ---------------------------------------------------------------- channel
def test_thermal_noise_floor_is_ktb():  # src/channel/mod.rs:342-350
    L = O.lib()
    p = L.orc_thermal_noise_power_w(290.0, 2.048e6)
    assert abs(p / (1.380649e-23 * 290.0 * 2.048e6) - 1) < 1e-12
    assert abs(10 * math.log10(p * 1e3) + 110.9) < 0.1
    assert L.orc_thermal_noise_power_w(580.0, 2.048e6) == 2 * p
    assert L.orc_thermal_noise_power_w(290.0, 4.096e6) == 2 * p


def _stationary(xyz):
    tr = O.Traj()
    tr.kind = 0
    tr.pos[0], tr.pos[1], tr.pos[2] = xyz
    return tr


def test_emission_solve_applies_sagnac():  # src/channel/mod.rs:355-383
    s = [25.0e6, 10.0e6, 0.0]
    obs = [6378137.0, 0.0, 0.0]
    tr = _stationary(s)
    o = np.array(obs, dtype=np.float64).reshape(3, 1).copy()
    t = np.zeros(1)
    te, rg = np.zeros(1), np.zeros(1)
    O.lib().orc_solve_emission_times(C.byref(tr), O.dptr(o), O.dptr(t), 1, 1717260840.0, 4, O.dptr(te), O.dptr(rg))
    solved = rg[0]
    naive = math.dist(s, obs)
    th = 7.2921151467e-5 * solved / SPEED_OF_LIGHT
    sr = [s[0] * math.cos(th) + s[1] * math.sin(th), -s[0] * math.sin(th) + s[1] * math.cos(th), s[2]]
    exact = math.dist(sr, obs)
    assert abs(solved - naive) > 1.0
    assert abs(solved - exact) < 0.01


def test_antenna_cutoff_occludes():  # src/channel/mod.rs:385-418
    obs = np.tile(np.array([[6378137.0], [0.0], [0.0]]), (1, 8)).copy()
    t = np.zeros(8)
    tx = _tx("ca_code", {"prn": 1, "epoch_unix": EPOCH, "nav": "off", "nav_seed": 0}, carrier=1575.42e6)
    sc, sig = _signal(tx)
    occ = O.Antenna(0.0, 0.0, 0.0, 0.0, 1)
    opn = O.Antenna(0.0, 0.0, 0.0, 0.0, 0)

    def power(pos, ant):
        tr = _stationary(pos)
        acc = np.zeros(16, dtype=np.float32)
        O.lib().orc_accumulate(O.fptr(acc), sig, C.byref(tr), O.dptr(obs), O.dptr(t), O.dptr(t), O.dptr(t), 8,
                               1575.42e6, 20.0, 1717260840.0, 4, C.byref(ant) if ant else None)
        return float(np.sum(acc.astype(np.float64) ** 2))

    above, below = [6.9e6, 0.0, 0.0], [-7.0e6, 0.0, 0.0]
    assert power(below, None) > 0
    assert power(below, opn) > 0
    assert power(below, occ) == 0.0
    assert power(above, occ) > 0


def test_bands_overlap_edges():  # src/pipeline.rs:1107-1141
    L = O.lib()
    lo, bw = 1_575_420_000.0, 2_048_000.0
    assert not L.orc_bands_overlap(437e6, 2 * 9600.0, lo, bw)
    assert L.orc_bands_overlap(lo, 2 * 1_023_000.0, lo, bw)
    edge = lo + bw / 2
    assert L.orc_bands_overlap(edge, 0.0, lo, bw)
    assert not L.orc_bands_overlap(edge + 1.0, 0.0, lo, bw)
    assert L.orc_bands_overlap(lo + 5e6, 20e6, lo, bw)


def test_truth_delay_matches_geometry():  # src/pipeline.rs:1145-1181
    tr = _stationary([7e6, 0.0, 0.0])
    o = np.array([[7e6], [0.0], [300000.0]]).copy()
    t = np.zeros(1)
    te, rg = np.zeros(1), np.zeros(1)
    O.lib().orc_solve_emission_times(C.byref(tr), O.dptr(o), O.dptr(t), 1, EPOCH, 4, O.dptr(te), O.dptr(rg))
    assert abs(rg[0] / SPEED_OF_LIGHT - 300000.0 / SPEED_OF_LIGHT) < 1e-9


# ---------------------------------------------------------------- signals
def test_prn1_first_ten_chips():  # src/signal/ca_code.rs:202-208
    assert list(O.ca_code(1)[:10]) == [-1, -1, 1, 1, -1, 1, 1, 1, 1, 1]


def test_every_prn_is_a_balanced_gold_code():  # IS-GPS-200 Gold codes: 512 ones / 511 zeros
    codes = np.stack([O.ca_code(p) for p in range(1, 33)]).astype(np.int64)
    assert all(abs(int(c.sum())) == 1 for c in codes)
    assert len({c.tobytes() for c in codes}) == 32


def test_nav_preamble_at_subframe_starts():  # src/signal/ca_code.rs:235-246
    L = O.lib()
    exp = [-1, 1, 1, 1, -1, 1, -1, -1]
    for sf in range(3):
        assert [L.orc_nav_bit_pm(12345, sf * 300 + k) for k in range(8)] == exp


def test_nav_payload_flips():  # src/signal/ca_code.rs:264-272
    L = O.lib()
    payload = [L.orc_nav_bit_pm(999, i) for i in range(8, 300)]
    assert 1 in payload and -1 in payload


def test_ca_pure_and_dummy_overlay():  # src/signal/ca_code.rs:210-262
    tx = _tx("ca_code", {"prn": 1, "epoch_unix": EPOCH, "nav": "off", "nav_seed": 0})
    sc, sig = _signal(tx)
    assert _eval(sig, [1e-9])[0].real == O.ca_code(1)[0]
    tx = _tx("ca_code", {"prn": 1, "epoch_unix": EPOCH, "nav": "dummy", "nav_seed": 42})
    sc, sig = _signal(tx)
    seed = (42 + 1 * 0xD1B54A32D192ED03) & 0xFFFFFFFFFFFFFFFF
    assert _eval(sig, [1e-9])[0].real == O.ca_code(1)[0] * O.lib().orc_nav_bit_pm(seed, 0)


def test_elapsed_periods_splits_exactly():  # src/signal/mod.rs:129-150
    assert O.elapsed_periods(1_717_260_840.0, 4800.0) == (8_242_852_032_000, 0.0)
    w, f = O.elapsed_periods(1_717_260_840.0 + 1.0 / 1_048_576.0, 4800.0)
    assert w == 8_242_852_032_000 and abs(f - 4800.0 / 1_048_576.0) < 1e-15
    assert O.elapsed_periods(-0.25, 2.0) == (-1, 0.5)
    rate = 9600.0 / 7.0
    w0, f0 = O.elapsed_periods(1.0e9, rate)
    w1, f1 = O.elapsed_periods(1.0e9 + 7.0, rate)
    assert w1 - w0 == 9600 and abs(f1 - f0) < 1e-9
    with pytest.raises(ValueError):
        O.elapsed_periods(float("inf"), 1.0)
    with pytest.raises(ValueError):
        O.elapsed_periods(1.0e12, 1.0e12)


def _bpsk(seed=11, n=59, rate=1000.0, sync=(-1, 1, 1, -1, 1), epoch=None):
    return _tx("bpsk", {"bit_rate_bps": rate, "payload_bits": n, "payload_seed": seed, "sync_word": list(sync)},
               carrier=401.15e6, signal_epoch_unix=epoch)


def test_anchored_bpsk_repeats():  # src/signal/mod.rs:170-198
    sc, f = _signal(_bpsk(epoch=1.0e9), render_epoch=1.0e9)
    n = f.contents.n
    assert n == 64
    bits = [f.contents.pm[i] for i in range(n)]
    for k in [-200, -65, -64, -1, 0, 1, 63, 64, 65, 1_000_003]:
        assert _eval(f, [(k + 0.5) * 1e-3])[0].real == bits[k % n]
    sc2, g = _signal(_bpsk(epoch=1.0e9 - 0.64 - 0.0025), render_epoch=1.0e9)
    assert g.contents.has_repeat == 1 and g.contents.repeat_from == 2
    assert abs(g.contents.epoch_rel_s + 0.0005) < 1.2e-7
    gb = [g.contents.pm[i] for i in range(64)]
    s = _eval(g, [0.0, 0.0003, 0.0007])
    assert [s[0].real, s[1].real, s[2].real] == [gb[2], gb[2], gb[3]]


def _same_from_two_epochs(make, rate):  # src/signal/mod.rs:152-168
    ea = 1_717_260_840.0
    shift = 1234.5
    sa, a = make(ea)
    sb, b = make(ea + shift)
    ta = np.array([shift - 1.0 + (k + 0.5) / rate for k in range(4000)])
    va, vb = _eval(a, ta), _eval(b, ta - shift)
    assert np.max(np.abs(va - vb)) < 1e-4
    assert np.any(np.abs(va) > 0.5)


def test_anchored_kinds_ignore_render_epoch():  # src/signal/mod.rs:200-224
    se = 1_000_000_007.25
    _same_from_two_epochs(lambda e: _signal(_bpsk(epoch=se), render_epoch=e), 1000.0)
    ook = _tx("ook", {"bit_rate_bps": 2400.0, "payload_bits": 93, "payload_seed": 5, "sync_word": [1, 0, 1, 1]},
              signal_epoch_unix=se)
    _same_from_two_epochs(lambda e: _signal(ook, render_epoch=e), 2400.0)
    qam = _tx("qam16", {"symbol_rate_baud": 1200.0, "payload_symbols": 30, "payload_seed": 6,
                        "sync_word": [1, 0, 1, 1]}, signal_epoch_unix=se)
    _same_from_two_epochs(lambda e: _signal(qam, render_epoch=e), 1200.0)
    cw = _tx("cw", {"baseband_offset_hz": 1234.5}, signal_epoch_unix=se)
    _same_from_two_epochs(lambda e: _signal(cw, render_epoch=e), 20000.0)
    ph = C.c_double()
    O.lib().orc_cw_anchor_phase(se, se, 1234.5, C.byref(ph))
    assert ph.value == 0.0


def test_cw_tone():  # src/signal/cw.rs:62-73
    sc, s = _signal(_tx("cw", {"baseband_offset_hz": 1000.0}, carrier=437e6))
    t = np.array([0.0, 0.25e-3, 0.5e-3, 0.7e-3, 1.0e-3])
    v = _eval(s, t)
    ph = 2 * math.pi * 1000.0 * t
    assert np.max(np.abs(v.real - np.cos(ph))) < 1e-5 and np.max(np.abs(v.imag - np.sin(ph))) < 1e-5


def test_qam16_constellation():  # src/signal/qam16.rs:129-161
    pts = []
    for v in range(16):
        sync = [(v >> 3) & 1, (v >> 2) & 1, (v >> 1) & 1, v & 1]
        sc, s = _signal(_tx("qam16", {"symbol_rate_baud": 1000.0, "payload_symbols": 0, "payload_seed": 0,
                                      "sync_word": sync}, carrier=2.4e9))
        pts.append((sync, _eval(s, [0.5e-3])[0]))
    levels = np.array([-3, -1, 1, 3]) / math.sqrt(10)
    for b, p in pts:
        assert np.min(np.abs(levels - p.real)) < 1e-6 and np.min(np.abs(levels - p.imag)) < 1e-6
    assert abs(np.mean([abs(p) ** 2 for _, p in pts]) - 1) < 1e-6
    step = 2 / math.sqrt(10)
    for ba, pa in pts:
        for bb, pb in pts:
            if abs(abs(pa - pb) - step) < 1e-5:
                assert sum(x != y for x, y in zip(ba, bb)) == 1


def test_qam16_frame_timing_and_payload():  # src/signal/qam16.rs:163-200
    sc, f = _signal(_tx("qam16", {"symbol_rate_baud": 2000.0, "payload_symbols": 4000, "payload_seed": 11,
                                  "sync_word": [0, 0, 0, 0, 1, 0, 1, 0]}, carrier=2.4e9))
    assert f.contents.n == 4002
    a = 3 / math.sqrt(10)
    s = _eval(f, [-1e-9, 0.0, 0.499e-3, 0.5e-3, 0.999e-3, 2001.0, 2001.5])
    assert s[0] == 0
    assert all(abs(s[i].real + a) < 1e-6 and abs(s[i].imag + a) < 1e-6 for i in (1, 2))
    assert all(abs(s[i].real - a) < 1e-6 and abs(s[i].imag - a) < 1e-6 for i in (3, 4))
    assert s[5] == 0 and s[6] == 0
    sym = np.ctypeslib.as_array(f.contents.sym, shape=(2 * 4002,)).view(np.complex64)[2:]
    assert abs(np.mean(np.abs(sym) ** 2) - 1) < 0.05
    assert len({(round(float(p.real), 4), round(float(p.imag), 4)) for p in sym}) == 16


def test_ook_frame():  # src/signal/ook.rs:87-119
    sync = [1, 0, 1, 1, 0, 0, 1, 0]
    sc, f = _signal(_tx("ook", {"bit_rate_bps": 1000.0, "payload_bits": 64, "payload_seed": 3,
                                "sync_word": sync}, carrier=433.92e6))
    n = f.contents.n
    bits = [f.contents.bits[i] for i in range(n)]
    assert n == 72 and bits[:8] == sync
    s = _eval(f, [(k + 0.5) * 1e-3 for k in range(n)])
    assert all(s[k] == complex(bits[k], 0) for k in range(n))
    ones = sum(bits[8:])
    assert 16 < ones < 48
    sc2, g = _signal(_tx("ook", {"bit_rate_bps": 1000.0, "payload_bits": 6, "payload_seed": 9,
                                 "sync_word": [1, 1]}, carrier=433.92e6))
    gb = [g.contents.bits[i] for i in range(8)]
    s = _eval(g, [-1e-6, 0.0, 7.999e-3, 8.0e-3, 1.0])
    assert s[0] == 0 and s[1] == 1 and s[2] == gb[7] and s[3] == 0 and s[4] == 0


def test_gate_intervals_and_anchoring():  # src/signal/gate.rs:118-164
    tx = _tx("cw", {"baseband_offset_hz": 50.0}, carrier=401.15e6,
             gate=cfg.Gate(15.0, [(0.0, 0.5), (1.5, 0.5), (3.0, 0.5)], epoch_unix=EPOCH))
    sc, g = _signal(tx)
    L = O.lib()
    for t, on in [(0.0, 1), (0.25, 1), (0.499999, 1), (0.5, 0), (1.0, 0), (1.499999, 0), (1.5, 1),
                  (1.999999, 1), (2.0, 0), (3.0, 1), (3.25, 1), (3.5, 0), (10.0, 0), (14.999999, 0)]:
        assert L.orc_gate_is_on(g, t) == on, t
    for k in [-3.0, -1.0, 1.0, 2.0, 1.0e6]:
        assert L.orc_gate_is_on(g, 15 * k + 0.25) and L.orc_gate_is_on(g, 15 * k + 1.75)
        assert not L.orc_gate_is_on(g, 15 * k + 0.75) and not L.orc_gate_is_on(g, 15 * k - 0.25)
    tx2 = _tx("cw", {"baseband_offset_hz": 50.0}, gate=cfg.Gate(15.0, [(0.0, 0.5), (1.5, 0.5), (3.0, 0.5)], 0.0))
    sc2, g2 = _signal(tx2, render_epoch=EPOCH + 4.0)
    assert not L.orc_gate_is_on(g2, 0.0) and not L.orc_gate_is_on(g2, 10.9)
    assert L.orc_gate_is_on(g2, 11.0) and L.orc_gate_is_on(g2, 11.4) and not L.orc_gate_is_on(g2, 11.5)
    assert L.orc_gate_is_on(g2, 12.5)


def test_gated_signal_zero_when_off():  # src/signal/gate.rs:166-191
    tx = _tx("cw", {"baseband_offset_hz": 50.0}, carrier=401.15e6,
             gate=cfg.Gate(15.0, [(0.0, 0.5), (1.5, 0.5), (3.0, 0.5)], epoch_unix=EPOCH))
    sc, g = _signal(tx)
    t = np.arange(2000) * 0.01
    v = _eval(g, t)
    on = np.array([O.lib().orc_gate_is_on(g, x) for x in t], dtype=bool)
    assert on.sum() == 300
    assert np.all(v[~on] == 0) and np.all(np.abs(v[on]) > 0.99)


# ---------------------------------------------------------------- rx chain
def _chain(**kw):
    fe = A.FrontendCfg(**kw)
    ch = O.RxChain()
    O.lib().orc_rx_chain_from_config(C.byref(fe), 1, C.byref(ch))
    return ch


def test_adc_quantises_and_clips():  # src/rx/mod.rs:171-193
    ch = _chain(has_adc=1, adc_bits=4, adc_full_scale_v=1.0)
    iq = np.array([0.5, -0.5, 2.0, -3.0], dtype=np.float32)
    O.lib().orc_rx_apply_post_sum(C.byref(ch), O.fptr(iq), 2)
    lsb = np.float32(1.0) / np.float32(7.0)
    for v in iq:
        assert abs(v) <= 1 + 1e-6 and abs(round(v / lsb) * lsb - v) < 1e-6
    assert iq[2] == 1.0 and iq[3] == -1.0


def test_antenna_pattern():  # src/rx/mod.rs:197-209
    a = O.Antenna(3.9, -3.0, 8.5, 0.0, 0)
    L = O.lib()
    g = lambda e: 20 * math.log10(L.orc_antenna_amplitude(C.byref(a), e))
    assert abs(g(90.0) - 3.9) < 1e-3 and abs(g(0.0) + 3.0) < 1e-3 and abs(g(-10.0) + 11.5) < 1e-3
    assert g(0.0) < g(45.0) < g(90.0)
    ac = O.Antenna(3.9, -3.0, 8.5, 0.0, 1)
    assert L.orc_antenna_amplitude(C.byref(ac), -0.1) == 0.0
    assert L.orc_antenna_amplitude(C.byref(ac), 0.0) > 0.0
    assert L.orc_antenna_amplitude(C.byref(ac), 45.0) == L.orc_antenna_amplitude(C.byref(a), 45.0)


def test_gain_and_nonlinearity():  # src/rx/mod.rs:211-245
    ch = _chain(has_gain=1, gain_db=20.0)
    iq = np.array([0.1, -0.2], dtype=np.float32)
    O.lib().orc_rx_apply_post_sum(C.byref(ch), O.fptr(iq), 1)
    assert abs(iq[0] - 1) < 1e-5 and abs(iq[1] + 2) < 1e-5
    ch = _chain(has_nonlinearity=1, iip3_dbm=0.0)
    iq = np.array([1e-4, 0.0, 0.02, 0.0], dtype=np.float32)
    O.lib().orc_rx_apply_post_sum(C.byref(ch), O.fptr(iq), 2)
    assert abs(iq[0] - 1e-4) / 1e-4 < 1e-3 and iq[2] < 0.02
    assert abs(iq[2] - 0.02 * (1 - (4 / 3) * 4e-4 / 1e-3)) < 1e-6


# ---------------------------------------------------------------- clock
def _clock(spec, rate, seed):
    cs = A.ClockCfg(*spec)
    return O.lib().orc_clock_new(C.byref(cs), 0.0, rate, seed)


def test_linear_drift_exact():  # src/clock/mod.rs:375-392
    h = _clock((0.0, 0.0, 5e-6, 0.0), 1e6, 42)
    last = O.lib().orc_clock_delta_t_at_master_index(h, 999_999)
    assert abs(last / (5e-6 * (1 - 1e-6)) - 1) < 1e-12
    O.lib().orc_clock_free(h)


def test_walk_is_cumulative_normal_increments():  # src/clock/mod.rs:424-444 (stream == materialised)
    L = O.lib()
    spec = (1e-11, 0.0, 0.5e-6, 1e-7)
    h = _clock(spec, 1e6, 123)
    rng = O.Xoshiro()
    L.orc_xoshiro_seed(C.byref(rng), 123)
    step = 1e-11 / math.sqrt(1e6)
    acc = 0.0
    for k in range(2000):
        acc += 0.0 + step * L.orc_std_normal(C.byref(rng))
        exp = acc + (1e-7 + 0.5e-6 * (k / 1e6))
        assert L.orc_clock_delta_t_at_master_index(h, k) == exp
    L.orc_clock_free(h)


def test_allan_deviation_recovers_target():  # src/clock/mod.rs:394-422
    L = O.lib()
    fs = 1e5
    h = _clock((1e-11, 0.0, 0.0, 0.0), fs, 7)
    step = int(fs)
    track = np.array([L.orc_clock_delta_t_at_master_index(h, k) for k in range(0, int(fs * 60) + 1, step)])
    L.orc_clock_free(h)
    d = np.diff(track)
    assert abs(np.std(d) / 1e-11 - 1) < 0.4


def test_clock_two_bands_coherent():  # src/clock/mod.rs:475-510
    L = O.lib()
    spec = (1e-11, 0.0, 0.3e-6, 0.0)
    master, low = 2.048e6, 48000.0
    hi = _clock(spec, master, 99)
    lo = _clock(spec, master, 99)
    n_hi = int(500 / low * master) + 2
    hv = np.array([L.orc_clock_delta_t_at(hi, i / master) for i in range(n_hi)])
    for j in range(500):
        t = j / low
        x = t * master
        k0 = int(math.floor(x))
        fr = x - k0
        ref = hv[k0] * (1 - fr) + hv[k0 + 1] * fr
        got = L.orc_clock_delta_t_at(lo, t)
        assert abs(got - ref) <= max(1e-9 * abs(ref), 1e-18)
    L.orc_clock_free(hi)
    L.orc_clock_free(lo)


def test_flicker_floor_flat():  # src/clock/mod.rs:355-373
    L = O.lib()
    fc = 128.0
    h = _clock((0.0, 1e-10, 0.0, 0.0), fc, 42)
    n = 1 << 18
    delta = np.array([L.orc_clock_delta_t_at_master_index(h, k) for k in range(n)])
    L.orc_clock_free(h)

    def adev(tau):
        m = int(tau * fc)
        d = delta[2 * m::m][: (n - 2 * m - 1) // m + 1]
        i = np.arange(0, n - 2 * m, m)
        dd = delta[i + 2 * m] - 2 * delta[i + m] + delta[i]
        return math.sqrt(np.mean(dd ** 2) / (2 * tau * tau))

    a1, a2, a8 = adev(1.0), adev(2.0), adev(8.0)
    assert 0.3e-10 < a2 < 3.0e-10
    assert 0.45 < a8 / a1 < 2.2


# ---------------------------------------------------------------- integration
def _run(text, seed, noise=O.NOISE_SEQUENTIAL, chunk=1 << 20, threads=1):
    return O.Scene(scenes.parse(text)).run(seed, chunk=chunk, threads=threads, noise=noise)


def test_clock_offset_survives_at_realistic_epoch():  # tests/multi_transmitter_summation.rs:134-157
    outs = dict(_run(scenes.CW_TWO_CLOCKS, 7))
    a, b = outs["rxb__b"].astype(np.complex128), outs["rxa__b"].astype(np.complex128)
    ph = np.angle(np.sum(a * np.conj(b)))
    rec = -ph / (2 * math.pi * 1e6)
    assert abs(rec - 1.3e-7) < 1e-9


def test_bpsk_radiates():  # tests/multi_transmitter_summation.rs:159-173
    iq = _run(scenes.BPSK, 1)[0][1]
    assert np.mean(np.abs(iq.astype(np.complex128)) ** 2) > 1e-13


def test_noise_only_power():  # tests/multi_transmitter_summation.rs:175-187
    iq = _run(scenes.NO_TX, 12345)[0][1]
    assert abs(np.mean(np.abs(iq.astype(np.complex128)) ** 2) / 1e-15 - 1) < 0.02


def test_superposition_one_noise_draw():  # tests/multi_transmitter_summation.rs:189-242
    both = scenes.parse(scenes.TWO_TX)
    alpha = both.clone()
    alpha.transmitters = [t for t in alpha.transmitters if t.name == "alpha"]
    beta = both.clone()
    beta.transmitters = [t for t in beta.transmitters if t.name == "beta"]
    run = lambda s: O.Scene(s).run(99, noise=O.NOISE_SEQUENTIAL)[0][1]
    a, b, ab, n = run(alpha), run(beta), run(both), run(scenes.parse(scenes.NO_TX))
    err = np.max(np.abs(ab - (a + b - n)))
    assert err < 1e-10


def _envelope(sig):
    iq = O.Scene(scenes.parse(scenes.OOK_QAM_TEMPLATE.replace("@SIGNAL@", sig))).run(1, noise=O.NOISE_SEQUENTIAL)[0][1]
    return np.abs(iq[1000:].astype(np.complex128)) ** 2


def test_ook_keys_between_off_and_cw():  # tests/ook_qam16_end_to_end.rs:451-468
    cw = np.mean(_envelope(scenes.SIG_CW))
    r = _envelope(scenes.SIG_OOK) / cw
    on = np.abs(r - 1) < 1e-3
    assert np.all(on | (r < 1e-6))
    assert abs(on.mean() - 0.5) < 0.05


def test_qam16_rings():  # tests/ook_qam16_end_to_end.rs:470-492
    cw = np.mean(_envelope(scenes.SIG_CW))
    r = _envelope(scenes.SIG_QAM16) / cw
    rings = np.array([0.2, 1.0, 1.8])
    k = np.argmin(np.abs(r[:, None] - rings[None, :]), axis=1)
    assert np.all(np.abs(r - rings[k]) < 1e-3)
    for i, e in enumerate([0.25, 0.5, 0.25]):
        assert abs(np.mean(k == i) - e) < 0.05
    assert abs(np.mean(r) - 1) < 0.05


def test_chunk_and_thread_invariance():  # tests/streaming_chunk_invariance.rs:320-391
    big = _run(scenes.STREAMING, 4242, chunk=1 << 22, threads=1)
    small = _run(scenes.STREAMING, 4242, chunk=4096, threads=3)
    for (na, a), (nb, b) in zip(big, small):
        assert na == nb and a.tobytes() == b.tobytes() and len(a) > 0
