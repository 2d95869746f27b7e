"""CPU checks of the C-ABI library: exports, host-side table building, the
host clock stream and argument validation. No GPU work is launched."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from lipika_b200 import build as B
from lipika_b200 import config as cfg
from lipika_b200 import native as N
from lipika_b200 import scene_abi as A
from oracle import oracle as O
from tests import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in ("lipika_cuda.h",):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(lpk_\w+)\s*\(", text):
            names.add(m.group(1))
    return names - {"lpk_sink_fn"}


def test_library_builds_and_exports_every_declared_symbol():
    B.build()
    L = C.CDLL(B.OUT)
    declared = _declared_functions()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert set(N.SIGNATURES) >= declared, sorted(declared - set(N.SIGNATURES))


def test_version_string():
    assert b"sm_100a" in N.lib().lpk_version()


class HostScene:
    """Host-side prepare without a device (tables only)."""

    def __init__(self, scene, time_base=A.LPK_TIME_BASE_SCENE, default_epoch=0.0):
        self.cs = cfg.to_c(scene, time_base, default_epoch)
        h = C.c_void_p()
        N.check(N.lib().lpk_scene_prepare(None, C.byref(self.cs.cfg), C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            N.lib().lpk_scene_free(self.h)

    def tx(self, i):
        d = N.TxDesc()
        N.check(N.lib().lpk_scene_tx_desc(self.h, i, C.byref(d)))
        return d


def _compare_tables(scene, time_base=A.LPK_TIME_BASE_SCENE, default_epoch=0.0):
    hs = HostScene(scene, time_base, default_epoch)
    os_ = O.Scene(scene, time_base, default_epoch)
    for i in range(len(scene.transmitters)):
        d = hs.tx(i)
        t = O.lib().orc_scene_traj(os_.h, i).contents
        s = O.lib().orc_scene_signal(os_.h, i).contents
        if t.kind == 0:
            assert d.traj_kind == 0 and list(d.stationary_ecef) == list(t.pos)
        else:
            assert d.traj_kind == 1 and d.grid_n == t.n and d.grid_t0_unix == t.t0_unix and d.grid_dt_s == t.dt_s
            a = np.ctypeslib.as_array(d.grid_xyz, shape=(3 * d.grid_n,))
            b = np.ctypeslib.as_array(t.grid, shape=(3 * t.n,))
            assert a.tobytes() == b.tobytes()
        assert d.sig_kind == s.kind and d.carrier_hz == s.carrier_hz
        assert d.tx_power_w == O.lib().orc_scene_tx_power_w(os_.h, i)
        if s.kind in (1, 2, 3):
            assert d.n_sym == s.n and d.epoch_rel_s == s.epoch_rel_s and d.has_repeat == s.has_repeat
            assert (not s.has_repeat) or d.repeat_from == s.repeat_from
            n = s.n
            if s.kind == 1:
                assert bytes(np.ctypeslib.as_array(d.pm_bits, (n,))) == bytes(np.ctypeslib.as_array(s.pm, (n,)))
            elif s.kind == 2:
                assert bytes(np.ctypeslib.as_array(d.ook_bits, (n,))) == bytes(np.ctypeslib.as_array(s.bits, (n,)))
            else:
                a = np.ctypeslib.as_array(C.cast(d.symbols, C.POINTER(C.c_float)), (2 * n,))
                b = np.ctypeslib.as_array(s.sym, (2 * n,))
                assert a.tobytes() == b.tobytes()
        elif s.kind == 4:
            assert bytes(np.ctypeslib.as_array(d.chips, (1023,))) == bytes(s.code)
            assert d.epoch_rel_s == s.epoch_rel_s and d.nav_kind == s.nav
            assert s.nav != 1 or d.nav_seed == s.nav_seed
        else:
            assert d.cw_anchored == s.cw_anchored and d.cw_phase0 == s.cw_phase0
            assert d.cw_offset_hz == s.cw_offset_hz
        assert d.has_gate == s.has_gate
        if s.has_gate:
            assert d.gate_period_s == s.gate_period_s and d.gate_phase_s == s.gate_phase_s
            assert d.gate_n == s.gate_n


def test_host_tables_match_oracle_c1():
    _compare_tables(scenes.config_c1(duration_s=5.0))


def test_host_tables_match_oracle_c4_all_kinds():
    _compare_tables(scenes.config_c4(duration_s=0.5, n_rx=1))


def test_host_tables_match_oracle_anchored_window_render():
    sc = scenes.config_c4(duration_s=0.5, n_rx=1)
    for t in sc.transmitters:
        if t.kind == "ca_code":
            t.params["nav"] = "off"
    sc.transmitters[0].gate = cfg.Gate(15.0, [(0.0, 0.5), (1.5, 0.5)], 7.0)
    _compare_tables(sc, A.LPK_TIME_BASE_ABSOLUTE, 0.0)


def test_host_clock_stream_matches_oracle_bit_for_bit():
    spec = A.ClockCfg(1e-9, 0.0, 0.5e-6, 1e-7)
    L = N.lib()
    h = C.c_void_p()
    N.check(L.lpk_clock_new(C.byref(spec), 0.0, 1e6, 4242, C.byref(h)))
    oc = O.lib().orc_clock_new(C.byref(spec), 0.0, 1e6, 4242)
    t = np.arange(50_000, dtype=np.float64) / 2.0e5
    got = np.zeros_like(t)
    N.check(L.lpk_clock_delta_t(h, N.dptr(t), len(t), N.dptr(got)))
    exp = np.array([O.lib().orc_clock_delta_t_at(oc, x) for x in t])
    L.lpk_clock_free(h)
    O.lib().orc_clock_free(oc)
    assert got.tobytes() == exp.tobytes()


def test_flicker_track_is_the_oracle_stream_flicker():
    """lpk_clock_flicker_table (the device clocks' flicker input) holds the
    oracle stream's flicker at the coarse points, and its linear
    interpolation (Flicker::delta_at, src/clock/mod.rs:142-148) reproduces the
    stream at every sample time, bit for bit."""
    spec = A.ClockCfg(0.0, 3e-10, 0.0, 0.0)
    L = N.lib()
    n = L.lpk_clock_flicker_len(5.0)
    assert n == 5 * 128 + 2
    tab = np.zeros(n)
    N.check(L.lpk_clock_flicker_table(C.byref(spec), 31, N.dptr(tab), n))
    oc = O.lib().orc_clock_new(C.byref(spec), 0.0, 48_000.0, 31)
    t = np.arange(0, 5 * 48_000, 7, dtype=np.float64) / 48_000.0
    exp = np.array([O.lib().orc_clock_delta_t_at(oc, x) for x in t])
    O.lib().orc_clock_free(oc)
    x = t * 128.0
    fl = np.floor(x)
    m = fl.astype(np.int64)
    frac = x - fl
    got = 0.0 + (tab[m] * (1.0 - frac) + tab[m + 1] * frac)  # (ε = 0 + flicker) + (c + m t = 0)
    assert got.tobytes() == (exp + 0.0).tobytes()
    assert np.std(np.diff(tab)) > 0.0
    bad = A.ClockCfg(1e-11, 0.0, 0.0, 0.0)
    assert L.lpk_clock_flicker_table(C.byref(bad), 31, N.dptr(tab), n) == N.LPK_EINVAL


def test_band_desc_carries_the_scene_flicker_track():
    sc = scenes.config_c0(duration_s=2.0, clock=cfg.Clock(allan_deviation_1s=1e-11, flicker_floor=2e-10))
    hs = HostScene(sc)

    def desc():
        d = N.BandDesc()
        N.check(N.lib().lpk_scene_band_desc(hs.h, 0, 0, 2026, 0, C.byref(d)))
        return d
    d = desc()
    assert d.flicker_n == 2 * 128 + 2 and bool(d.flicker_delta_s)
    tab = np.ctypeslib.as_array(d.flicker_delta_s, (d.flicker_n,)).copy()
    exp = np.zeros(d.flicker_n)
    spec = A.ClockCfg(1e-11, 2e-10, sc.receivers[0].clock.frequency_offset_y0,
                      sc.receivers[0].clock.initial_time_offset_s)
    N.check(N.lib().lpk_clock_flicker_table(C.byref(spec), d.clock_seed, N.dptr(exp), d.flicker_n))
    assert tab.tobytes() == exp.tobytes()
    assert C.addressof(desc().flicker_delta_s.contents) == C.addressof(d.flicker_delta_s.contents)  # one track


def test_band_desc_receiver_kinds():
    """A circular Keplerian receiver is positioned on the device
    (LPK_RX_KEPLER, its elements in the descriptor); a stationary one keeps
    its ECEF position."""
    from lipika_b200 import workloads as W
    sc = scenes.config_c1(duration_s=1.0)
    sc.receivers.append(cfg.Receiver("leo", W._kepler(7_000_000.0, 45.0, 10.0, 20.0), cfg.Clock(),
                                     [cfg.Band("l1", 1575.42e6, 2.048e6, 290.0, None)]))
    hs = HostScene(sc)
    d = N.BandDesc()
    N.check(N.lib().lpk_scene_band_desc(hs.h, 0, 0, 2026, 0, C.byref(d)))
    assert d.rx_kind == N.LPK_RX_STATIONARY
    N.check(N.lib().lpk_scene_band_desc(hs.h, 1, 0, 2026, 2, C.byref(d)))
    assert d.rx_kind == N.LPK_RX_KEPLER
    o = d.rx_orbit
    assert (o.semi_major_axis_m, o.inclination_deg, o.raan_deg, o.true_anomaly_deg_at_epoch) == (
        7_000_000.0, 45.0, 10.0, 20.0)


def test_host_clock_with_flicker_matches_oracle():
    spec = A.ClockCfg(0.0, 1e-10, 0.0, 0.0)
    L = N.lib()
    h = C.c_void_p()
    N.check(L.lpk_clock_new(C.byref(spec), 0.0, 1000.0, 9, C.byref(h)))
    oc = O.lib().orc_clock_new(C.byref(spec), 0.0, 1000.0, 9)
    t = np.arange(5000, dtype=np.float64) / 1000.0
    got = np.zeros_like(t)
    N.check(L.lpk_clock_delta_t(h, N.dptr(t), len(t), N.dptr(got)))
    exp = np.array([O.lib().orc_clock_delta_t_at(oc, x) for x in t])
    L.lpk_clock_free(h)
    O.lib().orc_clock_free(oc)
    assert got.tobytes() == exp.tobytes()


def test_host_rejects_what_the_reference_rejects():
    bad = scenes.config_c4(duration_s=0.1, n_rx=1)
    bad.transmitters[16].params["sync_word"] = [1, 0, 2]  # ook sync word not 0/1
    with pytest.raises(N.LpkError):
        HostScene(bad)
    bad = scenes.config_c4(duration_s=0.1, n_rx=1)
    bad.transmitters[32].params["sync_word"] = [1, 0, 1]  # qam16 partial symbol
    with pytest.raises(N.LpkError):
        HostScene(bad)
    bad = scenes.config_c1(duration_s=0.1)
    bad.transmitters[1].params["nav"] = "full"  # LNAV generation is out of scope
    with pytest.raises(N.LpkError) as e:
        HostScene(bad)
    assert e.value.code == N.LPK_ENOTSUP
    sc = scenes.config_c1(duration_s=0.1)
    sc.transmitters[1].params["nav"] = "dummy"
    with pytest.raises(N.LpkError):  # window render refuses a nav overlay
        HostScene(sc, A.LPK_TIME_BASE_ABSOLUTE, 0.0)
    g = scenes.config_c1(duration_s=0.1)
    g.transmitters[0].gate = cfg.Gate(15.0, [(14.8, 0.5)])
    with pytest.raises(N.LpkError):
        HostScene(g)


def test_band_descriptor_follows_reference_defaults():
    sc = scenes.config_c1(duration_s=1.0)
    hs = HostScene(sc)
    d = N.BandDesc()
    N.check(N.lib().lpk_scene_band_desc(hs.h, 0, 1, 2026, 1, C.byref(d)))
    assert d.noise_power_w == 1.380649e-23 * 290.0 * 2.048e6  # kTB, channel/mod.rs:310
    assert d.noise_seed == 2027                                # base + work_idx
    assert d.clock_seed == (2026 + 0xC10C000000000000) & 0xFFFFFFFFFFFFFFFF
    assert d.clock_mode == N.LPK_CLOCK_HOST and d.clock_master_rate_hz == 2.048e6
    act = (C.c_int32 * 16)()
    assert N.lib().lpk_scene_band_active(hs.h, 0, 0, act, 16) == 1 and act[0] == 0
    assert N.lib().lpk_scene_band_active(hs.h, 0, 1, act, 16) == 6
    assert N.lib().lpk_scene_band_samples(hs.h, 0, 1) == 2_048_000


def test_context_creation_fails_cleanly_without_a_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    h = C.c_void_p()
    code = N.lib().lpk_ctx_create(C.byref(h), 0)
    assert code != 0 and not h.value
    assert N.lib().lpk_global_last_error()


def test_config_parsing_defaults():
    sc = scenes.parse(scenes.STREAMING)
    assert sc.receivers[0].bands[0].noise_temperature_k == 290.0
    assert sc.transmitters[0].effective_bandwidth_hz() == 0.0
    sky = cfg.sky_from_toml_str("")
    assert sky.transmitters == [] and sky.gps_utc_offset_s == 18.0
    with pytest.raises(cfg.ConfigError):
        cfg.sky_from_toml_str("[scene]\nepoch_unix = 1.0\n")
    c1 = scenes.config_c1(1.0)
    assert c1.transmitters[0].effective_bandwidth_hz() == 2 * 9600.0
    assert c1.transmitters[1].effective_bandwidth_hz() == 2 * 1_023_000.0


def test_device_tables_flag_needs_a_context_and_known_flags():
    sc = scenes.config_c1(duration_s=0.1)
    cs = cfg.to_c(sc, A.LPK_TIME_BASE_SCENE, 0.0)
    h = C.c_void_p()
    cs.cfg.flags = A.LPK_SCENE_DEVICE_TABLES
    assert N.lib().lpk_scene_prepare(None, C.byref(cs.cfg), C.byref(h)) == N.LPK_EINVAL and not h.value
    cs.cfg.flags = 1 << 5
    assert N.lib().lpk_scene_prepare(None, C.byref(cs.cfg), C.byref(h)) == N.LPK_EINVAL and not h.value


def test_new_entry_points_reject_bad_arguments_without_a_gpu():
    L = N.lib()
    paths = (C.c_char_p * 1)(b"/nonexistent/x.iq.c64")
    assert L.lpk_generate_scene_to_files(None, 0, 1.0, 0, paths) == N.LPK_EINVAL
    o = (N.KeplerOrbit * 1)(N.KeplerOrbit(7e6, 50.0, 0.0, 0.0, 0.0))
    g = np.zeros(6)
    assert L.lpk_kepler_tables(None, o, 1, 0.0, 0.01, 2, g.ctypes.data_as(N._D)) == N.LPK_EINVAL
    assert L.lpk_sample_times(None, 2.048e6, 0, 4, g.ctypes.data_as(N._D)) == N.LPK_EINVAL
