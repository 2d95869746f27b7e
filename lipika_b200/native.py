"""ctypes binding of liblipika_cuda.so (include/lipika_cuda.h).

Loading never falls back to anything: if the in-tree library is missing or
fails to load, `lib()` raises, so no CPU path can stand in for the kernels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import scene_abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblipika_cuda.so")

LPK_OK = 0
LPK_EINVAL = -1
LPK_ENOMEM = -2
LPK_ECUDA = -3
LPK_ETIMEDOUT = -4
LPK_ENOCONV = -5
LPK_ENOTSUP = -6

LPK_TX_TRAJ_STATIONARY, LPK_TX_TRAJ_PRECOMPUTED = 0, 1
LPK_CLOCK_HOST, LPK_CLOCK_DETERMINISTIC, LPK_CLOCK_DEVICE_WALK = 0, 1, 2
LPK_RX_STATIONARY, LPK_RX_PER_SAMPLE = 0, 1
LPK_POST_GAIN, LPK_POST_NONLINEARITY, LPK_POST_ADC = 0, 1, 2
LPK_SOLVER_REFERENCE, LPK_SOLVER_SPLIT = 0, 1
LPK_NOISE_OFF, LPK_NOISE_ON, LPK_GEN_DEVICE_CLOCK, LPK_GEN_SPLIT = 0, 1, 2, 4


class LpkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lipika_cuda error {code}: {msg}")
        self.code = code


class CF32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class TxDesc(C.Structure):
    _fields_ = [
        ("traj_kind", C.c_int32), ("sig_kind", C.c_int32),
        ("stationary_ecef", C.c_double * 3),
        ("grid_t0_unix", C.c_double), ("grid_dt_s", C.c_double), ("grid_n", C.c_int64),
        ("grid_xyz", C.POINTER(C.c_double)),
        ("carrier_hz", C.c_double), ("tx_power_w", C.c_double),
        ("epoch_rel_s", C.c_double), ("rate_hz", C.c_double),
        ("has_repeat", C.c_int32), ("nav_kind", C.c_int32),
        ("repeat_from", C.c_int64), ("n_sym", C.c_int64),
        ("pm_bits", C.POINTER(C.c_int8)), ("ook_bits", C.POINTER(C.c_uint8)),
        ("symbols", C.POINTER(CF32)), ("chips", C.POINTER(C.c_int8)),
        ("nav_seed", C.c_uint64), ("nav_bits", C.POINTER(C.c_int8)), ("nav_n", C.c_int64),
        ("cw_offset_hz", C.c_double), ("cw_phase0", C.c_double),
        ("cw_anchored", C.c_int32), ("has_gate", C.c_int32),
        ("gate_period_s", C.c_double), ("gate_phase_s", C.c_double),
        ("gate_n", C.c_int32), ("reserved", C.c_int32),
        ("gate_on", C.POINTER(C.c_double)),
    ]


class PostOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("bits", C.c_uint32), ("param", C.c_double)]


class BandDesc(C.Structure):
    _fields_ = [
        ("epoch_unix", C.c_double), ("fs_hz", C.c_double), ("lo_hz", C.c_double),
        ("noise_power_w", C.c_double), ("noise_seed", C.c_uint64),
        ("rx_kind", C.c_int32), ("clock_mode", C.c_int32),
        ("rx_ecef", C.c_double * 3),
        ("clock_offset_s", C.c_double), ("clock_y0", C.c_double),
        ("clock_allan_1s", C.c_double), ("clock_master_rate_hz", C.c_double),
        ("clock_seed", C.c_uint64),
        ("has_antenna", C.c_int32), ("has_cutoff", C.c_int32),
        ("ant_peak_dbi", C.c_double), ("ant_horizon_dbi", C.c_double),
        ("ant_fb_db", C.c_double), ("ant_cutoff_deg", C.c_double),
        ("n_post", C.c_int32), ("solver", C.c_int32),
        ("post", PostOp * 3),
    ]


class BandResult(C.Structure):
    _fields_ = [("n_samples", C.c_int64), ("stopped_early", C.c_int32), ("n_active", C.c_int32),
                ("unoccluded", C.c_uint8 * 256)]


SINK_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(CF32), C.c_int64)

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_CF = C.POINTER(CF32)
_VP = C.c_void_p

# name -> (restype, argtypes); every entry point of include/lipika_cuda.h
SIGNATURES = {
    "lpk_ctx_create": (C.c_int32, [C.POINTER(_VP), C.c_int32]),
    "lpk_ctx_destroy": (None, [_VP]),
    "lpk_last_error": (C.c_char_p, [_VP]),
    "lpk_global_last_error": (C.c_char_p, []),
    "lpk_version": (C.c_char_p, []),
    "lpk_ctx_stream": (_VP, [_VP]),
    "lpk_profile_enable": (C.c_int32, [_VP, C.c_int32]),
    "lpk_profile_reset": (C.c_int32, [_VP]),
    "lpk_profile_read": (C.c_int32, [_VP, _D, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "lpk_probe_fp64_peak": (C.c_int32, [_VP, _D]),
    "lpk_scene_upload": (C.c_int32, [_VP, C.POINTER(TxDesc), C.c_int32]),
    "lpk_band_chunk": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64, _D, _D, _CF, _U8]),
    "lpk_band_chunk_device": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64,
                                          _VP, _VP, _VP, _VP]),
    "lpk_sync": (C.c_int32, [_VP]),
    "lpk_band_chunk_device_static": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64,
                                                 _VP, _VP, _VP, _VP]),
    "lpk_solve_emission_times": (C.c_int32, [_VP, C.c_int32, _D, _D, C.c_int64, C.c_double, C.c_int32, _D, _D]),
    "lpk_tx_contribution": (C.c_int32, [_VP, C.POINTER(BandDesc), C.c_int32, C.c_int64, C.c_int64, _D, _D, _CF,
                                        _D, _D, _D]),
    "lpk_clock_device_delta": (C.c_int32, [_VP, C.POINTER(BandDesc), C.c_int64, C.c_int64, _D]),
    "lpk_rx_chain_apply": (C.c_int32, [_VP, C.POINTER(BandDesc), _CF, C.c_int64]),
    "lpk_scene_prepare": (C.c_int32, [_VP, C.POINTER(A.SceneCfg), C.POINTER(_VP)]),
    "lpk_scene_free": (None, [_VP]),
    "lpk_scene_n_work": (C.c_int32, [_VP]),
    "lpk_scene_work": (C.c_int32, [_VP, C.c_int32, _I32, _I32]),
    "lpk_scene_band_samples": (C.c_int64, [_VP, C.c_int32, C.c_int32]),
    "lpk_scene_band_active": (C.c_int32, [_VP, C.c_int32, C.c_int32, _I32, C.c_int32]),
    "lpk_scene_tx_desc": (C.c_int32, [_VP, C.c_int32, C.POINTER(TxDesc)]),
    "lpk_scene_band_desc": (C.c_int32, [_VP, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.POINTER(BandDesc)]),
    "lpk_generate_band": (C.c_int32, [_VP, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int64, C.c_int32,
                                      SINK_FN, _VP, C.POINTER(BandResult)]),
    "lpk_generate_band_to_file": (C.c_int32, [_VP, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int64,
                                              C.c_int32, C.c_char_p, C.POINTER(BandResult)]),
    "lpk_clock_new": (C.c_int32, [C.POINTER(A.ClockCfg), C.c_double, C.c_double, C.c_uint64, C.POINTER(_VP)]),
    "lpk_clock_delta_t": (C.c_int32, [_VP, _D, C.c_int64, _D]),
    "lpk_clock_free": (None, [_VP]),
}

_lib = None


def lib():
    """Load the in-tree library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lipika_b200.build` "
                               "(the CUDA backend has no fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, ctx=None):
    if code != LPK_OK:
        L = lib()
        msg = (L.lpk_last_error(ctx) if ctx else b"") or L.lpk_global_last_error() or b""
        raise LpkError(code, msg.decode(errors="replace"))


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class Context:
    """An lpk_ctx: one CUDA device, its stream and its uploaded scene."""

    def __init__(self, device: int = 0):
        h = _VP()
        check(lib().lpk_ctx_create(C.byref(h), device))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().lpk_ctx_destroy(self.h)
            except Exception:  # interpreter shutdown
                pass
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, code):
        check(code, self.h)
