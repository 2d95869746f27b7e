"""ctypes wrapper of the CPU ORACLE (liblpk_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use it as the checker or the timed CPU baseline. The
product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from lipika_b200 import config as cfgmod
from lipika_b200 import scene_abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblpk_oracle.so")
_lib = None

NOISE_NONE, NOISE_COUNTER, NOISE_SEQUENTIAL = 0, 1, 2


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(_HERE, "lpk_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "liblpk_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


class Traj(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("n", C.c_int64),
                ("pos", C.c_double * 3), ("t0_unix", C.c_double), ("dt_s", C.c_double),
                ("grid", C.POINTER(C.c_double)), ("max_speed_m_s", C.c_double),
                ("max_radius_m", C.c_double), ("raw", A.TrajectoryCfg)]


class Signal(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nav", C.c_int32), ("carrier_hz", C.c_double),
                ("epoch_rel_s", C.c_double), ("rate_hz", C.c_double),
                ("has_repeat", C.c_int32), ("cw_anchored", C.c_int32),
                ("repeat_from", C.c_int64), ("n", C.c_int64),
                ("pm", C.POINTER(C.c_int8)), ("bits", C.POINTER(C.c_uint8)),
                ("sym", C.POINTER(C.c_float)), ("code", C.c_int8 * 1023),
                ("nav_seed", C.c_uint64), ("nav_bits", C.POINTER(C.c_int8)), ("nav_n", C.c_int64),
                ("cw_offset_hz", C.c_double), ("cw_phase0", C.c_double),
                ("has_gate", C.c_int32), ("gate_n", C.c_int32),
                ("gate_period_s", C.c_double), ("gate_phase_s", C.c_double),
                ("gate_on", C.POINTER(C.c_double))]


class Antenna(C.Structure):
    _fields_ = [("peak_dbi", C.c_double), ("horizon_dbi", C.c_double), ("fb_db", C.c_double),
                ("cutoff_deg", C.c_double), ("has_cutoff", C.c_int32), ("reserved", C.c_int32)]


class PostOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("bits", C.c_uint32), ("a", C.c_double)]


class RxChain(C.Structure):
    _fields_ = [("has_antenna", C.c_int32), ("n_post", C.c_int32), ("antenna", Antenna),
                ("post", PostOp * 3)]


class Xoshiro(C.Structure):
    _fields_ = [("s", C.c_uint64 * 4)]


_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_xoshiro_seed": (None, [C.POINTER(Xoshiro), C.c_uint64]),
            "orc_xoshiro_next": (C.c_uint64, [C.POINTER(Xoshiro)]),
            "orc_gen_bool_half": (C.c_int, [C.POINTER(Xoshiro)]),
            "orc_gen_range_u8_16": (C.c_uint32, [C.POINTER(Xoshiro)]),
            "orc_std_normal": (C.c_double, [C.POINTER(Xoshiro)]),
            "orc_philox4x32_10": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "orc_noise_pair": (None, [C.c_uint64, C.c_int64, _F, _F]),
            "orc_geodetic_to_ecef": (None, [C.c_double, C.c_double, C.c_double, _D]),
            "orc_kepler_position_ecef": (None, [C.POINTER(A.TrajectoryCfg), C.c_double, _D]),
            "orc_traj_sample": (C.c_int, [C.POINTER(A.TrajectoryCfg), C.c_double, C.c_double, C.c_double, C.POINTER(Traj)]),
            "orc_traj_for_transmitter": (C.c_int, [C.POINTER(A.TrajectoryCfg), C.c_double, C.c_double, C.POINTER(Traj)]),
            "orc_traj_position": (None, [C.POINTER(Traj), C.c_double, _D]),
            "orc_traj_position_batch": (None, [C.POINTER(Traj), _D, C.c_int64, _D]),
            "orc_traj_free": (None, [C.POINTER(Traj)]),
            "orc_elapsed_periods": (C.c_int, [C.c_double, C.c_double, C.POINTER(C.c_int64), _D]),
            "orc_frame_anchor": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int64, _D, C.POINTER(C.c_int64)]),
            "orc_cw_anchor_phase": (C.c_int, [C.c_double, C.c_double, C.c_double, _D]),
            "orc_ca_code": (None, [C.c_int, C.POINTER(C.c_int8)]),
            "orc_nav_bit_pm": (C.c_int8, [C.c_uint64, C.c_int64]),
            "orc_signal_build": (C.c_int, [C.POINTER(A.TransmitterCfg), C.POINTER(A.SceneCfg), C.POINTER(Signal)]),
            "orc_signal_eval": (None, [C.POINTER(Signal), _D, C.c_int64, _F]),
            "orc_gate_is_on": (C.c_int, [C.POINTER(Signal), C.c_double]),
            "orc_signal_free": (None, [C.POINTER(Signal)]),
            "orc_antenna_amplitude": (C.c_float, [C.POINTER(Antenna), C.c_double]),
            "orc_solve_emission_times": (None, [C.POINTER(Traj), _D, _D, C.c_int64, C.c_double, C.c_int, _D, _D]),
            "orc_solve_converged": (None, [C.POINTER(Traj), _D, _D, C.c_int64, C.c_double, C.c_double, C.c_int, _D, _D, C.POINTER(C.c_int32)]),
            "orc_accumulate": (C.c_int, [_F, C.POINTER(Signal), C.POINTER(Traj), _D, _D, _D, _D, C.c_int64,
                                         C.c_double, C.c_double, C.c_double, C.c_int, C.POINTER(Antenna)]),
            "orc_thermal_noise_power_w": (C.c_double, [C.c_double, C.c_double]),
            "orc_bands_overlap": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double]),
            "orc_rx_chain_from_config": (None, [C.POINTER(A.FrontendCfg), C.c_int, C.POINTER(RxChain)]),
            "orc_rx_apply_post_sum": (None, [C.POINTER(RxChain), _F, C.c_int64]),
            "orc_adc_codes": (C.c_int, [C.POINTER(RxChain), _F, C.c_int64, C.POINTER(C.c_int32)]),
            "orc_clock_new": (C.c_void_p, [C.POINTER(A.ClockCfg), C.c_double, C.c_double, C.c_uint64]),
            "orc_clock_delta_t_at": (C.c_double, [C.c_void_p, C.c_double]),
            "orc_clock_delta_t_at_master_index": (C.c_double, [C.c_void_p, C.c_int64]),
            "orc_clock_free": (None, [C.c_void_p]),
            "orc_clock_seed": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_noise_seed": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_scene_prepare": (C.c_int, [C.POINTER(A.SceneCfg), C.POINTER(C.c_void_p)]),
            "orc_scene_free": (None, [C.c_void_p]),
            "orc_scene_n_work": (C.c_int, [C.c_void_p]),
            "orc_scene_work": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "orc_band_n_samples": (C.c_int64, [C.c_void_p, C.c_int, C.c_int]),
            "orc_band_active": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32), C.c_int]),
            "orc_scene_signal": (C.POINTER(Signal), [C.c_void_p, C.c_int]),
            "orc_scene_traj": (C.POINTER(Traj), [C.c_void_p, C.c_int]),
            "orc_scene_tx_power_w": (C.c_double, [C.c_void_p, C.c_int]),
            "orc_generate_band": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int64, C.c_int,
                                            C.c_int, C.c_int64, _F, _D, C.POINTER(C.c_uint8)]),
            "orc_profile_sections": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int64, _D]),
            "orc_generate_band_window": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int64,
                                                   C.c_int, C.c_int, C.c_int64, C.c_int64, _F, _D,
                                                   C.POINTER(C.c_uint8)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


# ---------------------------------------------------------------- helpers
def geodetic_to_ecef(lat, lon, h):
    out = np.zeros(3)
    lib().orc_geodetic_to_ecef(lat, lon, h, dptr(out))
    return out


def ca_code(prn: int) -> np.ndarray:
    out = np.zeros(1023, dtype=np.int8)
    lib().orc_ca_code(prn, out.ctypes.data_as(C.POINTER(C.c_int8)))
    return out


def elapsed_periods(elapsed, rate):
    w = C.c_int64()
    f = C.c_double()
    rc = lib().orc_elapsed_periods(elapsed, rate, C.byref(w), C.byref(f))
    if rc:
        raise ValueError("symbol count is not representable")
    return w.value, f.value


class Scene:
    """Oracle-prepared scene (prepare, src/pipeline.rs:801-819)."""

    def __init__(self, scene: cfgmod.Scene, time_base=A.LPK_TIME_BASE_SCENE, default_signal_epoch_unix=0.0):
        self.cs = cfgmod.to_c(scene, time_base, default_signal_epoch_unix)
        h = C.c_void_p()
        rc = lib().orc_scene_prepare(C.byref(self.cs.cfg), C.byref(h))
        if rc:
            raise ValueError(f"oracle scene prepare failed ({rc})")
        self.h = h
        self.scene = scene

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_free(self.h)
            self.h = None

    def work(self):
        L = lib()
        out = []
        for w in range(L.orc_scene_n_work(self.h)):
            r, b = C.c_int(), C.c_int()
            L.orc_scene_work(self.h, w, C.byref(r), C.byref(b))
            out.append((r.value, b.value))
        return out

    def n_samples(self, r, b):
        return lib().orc_band_n_samples(self.h, r, b)

    def active(self, r, b):
        buf = (C.c_int32 * 256)()
        k = lib().orc_band_active(self.h, r, b, buf, 256)
        return [buf[i] for i in range(k)]

    def generate_band(self, r, b, seed, work_idx, chunk=1 << 20, threads=1, noise=NOISE_NONE,
                      limit=-1, want_delta=False):
        n = self.n_samples(r, b)
        if limit >= 0:
            n = min(n, limit)
        out = np.zeros(2 * max(n, 1), dtype=np.float32)
        delta = np.zeros(max(n, 1)) if want_delta else None
        na = len(self.active(r, b))
        unocc = (C.c_uint8 * max(na, 1))()
        rc = lib().orc_generate_band(self.h, r, b, seed, work_idx, chunk, threads, noise, limit,
                                     fptr(out), dptr(delta) if want_delta else None, unocc)
        if rc:
            raise RuntimeError(f"oracle generate_band failed ({rc})")
        iq = out[: 2 * n].view(np.complex64)
        res = {"iq": iq, "unoccluded": [bool(unocc[i]) for i in range(na)]}
        if want_delta:
            res["delta"] = delta[:n]
        return res

    def generate_window(self, r, b, seed, work_idx, start, n, chunk=1 << 20, threads=1, noise=NOISE_NONE):
        """Band samples [start, start + n) through the same loop (chunks
        begin at `start`); noise NONE or COUNTER."""
        n = max(0, min(n, self.n_samples(r, b) - start))
        out = np.zeros(2 * max(n, 1), dtype=np.float32)
        na = len(self.active(r, b))
        unocc = (C.c_uint8 * max(na, 1))()
        rc = lib().orc_generate_band_window(self.h, r, b, seed, work_idx, chunk, threads, noise, start, n,
                                            fptr(out), None, unocc)
        if rc:
            raise RuntimeError(f"oracle generate_band_window failed ({rc})")
        return out[: 2 * n].view(np.complex64)

    def profile_sections(self, r, b, seed, n):
        """Single-thread ns per sample of each section of the loop on the
        first n samples of band (r, b): clock, rx, solve, baseband, mix,
        sum, awgn, and the largest carrier-phase argument (rad)."""
        out = np.zeros(8)
        if lib().orc_profile_sections(self.h, r, b, seed, n, dptr(out)):
            raise RuntimeError("oracle profile failed")
        keys = ("clock_ns_per_band_sample", "rx_ns_per_band_sample", "solve_ns_per_txrx", "baseband_ns_per_txrx",
                "mix_ns_per_txrx", "sum_ns_per_band_sample", "awgn_ns_per_band_sample", "max_phase_rad")
        return dict(zip(keys, out.tolist()))

    def run(self, seed, chunk=1 << 20, threads=1, noise=NOISE_NONE):
        """run_scene (src/pipeline.rs:443-485): every (rx, band) in order."""
        outs = []
        for w, (r, b) in enumerate(self.work()):
            rx = self.scene.receivers[r]
            outs.append((f"{rx.name}__{rx.bands[b].band_id}",
                         self.generate_band(r, b, seed, w, chunk, threads, noise)["iq"]))
        return outs
