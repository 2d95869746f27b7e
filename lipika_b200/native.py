"""ctypes binding of liblipika_cuda.so (include/lipika_cuda.h).

Loading never falls back to anything: if the in-tree library is missing or
fails to load, `lib()` raises, so no CPU path can stand in for the kernels.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

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
LPK_RX_STATIONARY, LPK_RX_PER_SAMPLE, LPK_RX_KEPLER = 0, 1, 2
LPK_POST_GAIN, LPK_POST_NONLINEARITY, LPK_POST_ADC = 0, 1, 2
LPK_SOLVER_REFERENCE, LPK_SOLVER_SPLIT, LPK_SOLVER_FP64_TUNED = 0, 1, 2
LPK_NOISE_OFF, LPK_NOISE_ON, LPK_GEN_DEVICE_CLOCK, LPK_GEN_SPLIT, LPK_GEN_AUTOTUNE = 0, 1, 2, 4, 8
LPK_START_LAG, LPK_START_GEOMETRIC, LPK_START_LEARNED = 0, 1, 2
LPK_ITER_FIXED_POINT, LPK_ITER_NEWTON = 0, 1
MLP_N_FEATURES, MLP_N_PARAMS, MLP_N_NORM = 16, 9473, 34


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


class KeplerOrbit(C.Structure):
    _fields_ = [("semi_major_axis_m", C.c_double), ("inclination_deg", C.c_double), ("raan_deg", C.c_double),
                ("true_anomaly_deg_at_epoch", C.c_double), ("epoch_unix", C.c_double)]


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
        ("flicker_delta_s", C.POINTER(C.c_double)), ("flicker_n", C.c_int64),
        ("rx_orbit", KeplerOrbit),
    ]


class BandResult(C.Structure):
    _fields_ = [("n_samples", C.c_int64), ("stopped_early", C.c_int32), ("n_active", C.c_int32),
                ("unoccluded", C.c_uint8 * 256)]


class WorkUnit(C.Structure):
    _fields_ = [("band", BandDesc), ("active", C.POINTER(C.c_int32)), ("n_active", C.c_int32),
                ("reserved", C.c_int32), ("n_samples", C.c_int64)]


SINK_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(CF32), C.c_int64)
UNIT_SINK_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32, C.POINTER(CF32), C.c_int64)

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_CF = C.POINTER(CF32)
_F = C.POINTER(C.c_float)
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
    "lpk_gate_stats": (C.c_int32, [_VP, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int32]),
    "lpk_scene_upload": (C.c_int32, [_VP, C.POINTER(TxDesc), C.c_int32]),
    "lpk_generate_scene_to_files": (C.c_int32, [_VP, C.c_uint64, C.c_double, C.c_int32,
                                                 C.POINTER(C.c_char_p)]),
    "lpk_sample_times": (C.c_int32, [_VP, C.c_double, C.c_int64, C.c_int64, _D]),
    "lpk_kepler_tables": (C.c_int32, [_VP, C.POINTER(KeplerOrbit), C.c_int32, C.c_double, C.c_double, C.c_int64,
                                      _D]),
    "lpk_band_chunk": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64, _D, _D, _CF, _U8]),
    "lpk_band_chunk_device": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64,
                                          _VP, _VP, _VP, _VP]),
    "lpk_sync": (C.c_int32, [_VP]),
    "lpk_split_accuracy": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64, _VP, _VP,
                                       _D, _D, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "lpk_band_chunk_device_static": (C.c_int32, [_VP, C.POINTER(BandDesc), _I32, C.c_int32, C.c_int64, C.c_int64,
                                                 _VP, _VP, _VP, _VP]),
    "lpk_solve_emission_times": (C.c_int32, [_VP, C.c_int32, _D, _D, C.c_int64, C.c_double, C.c_int32, _D, _D]),
    "lpk_tx_contribution": (C.c_int32, [_VP, C.POINTER(BandDesc), C.c_int32, C.c_int64, C.c_int64, _D, _D, _CF,
                                        _D, _D, _D]),
    "lpk_clock_device_delta": (C.c_int32, [_VP, C.POINTER(BandDesc), C.c_int64, C.c_int64, _D]),
    "lpk_rx_chain_apply": (C.c_int32, [_VP, C.POINTER(BandDesc), _CF, C.c_int64]),
    "lpk_split_variant_count": (C.c_int32, []),
    "lpk_split_variant_info": (C.c_int32, [C.c_int32, _I32, _I32, _I32]),
    "lpk_ctx_set_split_variant": (C.c_int32, [_VP, C.c_int32]),
    "lpk_ctx_split_variant": (C.c_int32, [_VP]),
    "lpk_batch_create": (C.c_int32, [_VP, C.POINTER(WorkUnit), C.c_int32, C.c_double, C.POINTER(_VP)]),
    "lpk_batch_destroy": (None, [_VP]),
    "lpk_batch_n_rounds": (C.c_int64, [_VP]),
    "lpk_batch_round_extent": (C.c_int32, [_VP, C.c_int64, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "lpk_batch_run": (C.c_int32, [_VP, C.c_int64]),
    "lpk_batch_output": (C.c_int32, [_VP, C.c_int32, C.POINTER(_VP)]),
    "lpk_batch_copy_out": (C.c_int32, [_VP, C.c_int32, _CF, C.c_int64]),
    "lpk_batch_reset": (C.c_int32, [_VP]),
    "lpk_batch_render": (C.c_int32, [_VP, UNIT_SINK_FN, _VP]),
    "lpk_batch_set_config": (C.c_int32, [_VP, C.c_int32, C.c_int32]),
    "lpk_batch_get_config": (C.c_int32, [_VP, _I32, _I32, _I32]),
    "lpk_batch_autotune": (C.c_int32, [_VP, C.c_int64, C.c_int32, _D]),
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
    "lpk_generate_scene": (C.c_int32, [_VP, C.c_uint64, C.c_double, C.c_int32, UNIT_SINK_FN, _VP]),
    "lpk_solve_converged": (C.c_int32, [_VP, C.c_int32, _D, C.c_double, _D, C.c_int64, C.c_double, C.c_int32,
                                        C.c_int32, C.c_int32, _VP, _D, _I32, _F]),
    "lpk_solve_converged_scene": (C.c_int32, [_VP, _I32, _I32, _D, C.c_int32, C.c_double, _D, C.c_int64,
                                              C.c_double, C.c_int32, C.c_int32, C.c_int32, _VP, _D, _I32, _F, _D]),
    "lpk_mlp_features": (C.c_int32, [_VP, C.c_int32, _D, C.c_double, _D, C.c_int64, _F]),
    "lpk_mlp_set_orbits": (C.c_int32, [_VP, _I32, C.POINTER(KeplerOrbit), C.c_int32]),
    "lpk_mlp_wait_selftest": (C.c_int32, [_VP, C.c_int64, C.c_int32]),
    "lpk_mlp_create": (C.c_int32, [_VP, C.c_uint64, C.POINTER(_VP)]),
    "lpk_mlp_destroy": (None, [_VP]),
    "lpk_mlp_get_params": (C.c_int32, [_VP, _F, _F]),
    "lpk_mlp_set_params": (C.c_int32, [_VP, _F, _F]),
    "lpk_mlp_forward": (C.c_int32, [_VP, _F, C.c_int64, _F]),
    "lpk_mlp_loss_grad": (C.c_int32, [_VP, _F, _F, C.c_int64, _D, _F]),
    "lpk_mlp_fit": (C.c_int32, [_VP, _I32, C.POINTER(KeplerOrbit), C.c_int32, _D, C.c_int32, C.c_double,
                                C.c_double, C.c_double, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _F]),
    "lpk_clock_new": (C.c_int32, [C.POINTER(A.ClockCfg), C.c_double, C.c_double, C.c_uint64, C.POINTER(_VP)]),
    "lpk_clock_delta_t": (C.c_int32, [_VP, _D, C.c_int64, _D]),
    "lpk_clock_flicker_len": (C.c_int64, [C.c_double]),
    "lpk_clock_flicker_table": (C.c_int32, [C.POINTER(A.ClockCfg), C.c_uint64, _D, C.c_int64]),
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
    """An lpk_ctx: one CUDA device, its stream and its uploaded scene.

    Objects made on a context (a scene, a batch, a network) register here
    and are closed before the context itself: their C handles refer to it."""

    def __init__(self, device: int = 0):
        h = _VP()
        check(lib().lpk_ctx_create(C.byref(h), device))
        self.h = h
        self.device = device
        self._deps = weakref.WeakSet()

    def adopt(self, obj):
        """Close obj (it has a close()) before this context closes."""
        self._deps.add(obj)

    def close(self):
        for d in list(getattr(self, "_deps", ())):
            d.close()
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


def split_variants():
    """[(tile, threads, min_blocks)] of every compiled split launch shape."""
    L = lib()
    out = []
    for v in range(L.lpk_split_variant_count()):
        t, n, m = C.c_int32(), C.c_int32(), C.c_int32()
        check(L.lpk_split_variant_info(v, C.byref(t), C.byref(n), C.byref(m)))
        out.append((t.value, n.value, m.value))
    return out


class Batch:
    """An lpk_batch: work units (band descriptor, active list, length) of a
    scene rendered together, one graph-replayed round at a time."""

    def __init__(self, ctx: Context, units, round_s: float):
        """units: iterable of (BandDesc, active int sequence, n_samples)."""
        self.ctx = ctx
        self._act = []
        arr = (WorkUnit * len(units))()
        for k, (band, active, n) in enumerate(units):
            a = np.ascontiguousarray(np.asarray(active, dtype=np.int32))
            self._act.append(a)
            arr[k].band = band
            arr[k].active = a.ctypes.data_as(_I32) if a.size else None
            arr[k].n_active = int(a.size)
            arr[k].n_samples = int(n)
        h = _VP()
        ctx.check(lib().lpk_batch_create(ctx.h, arr, len(units), float(round_s), C.byref(h)))
        self.h = h
        ctx.adopt(self)
        self.n_units = len(units)
        self.n_rounds = int(lib().lpk_batch_n_rounds(h))
        self._caps = [max([self.extent(r, u)[1] for r in range(min(self.n_rounds, 2))] + [1])
                      for u in range(self.n_units)]

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().lpk_batch_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.close()

    def extent(self, rnd: int, unit: int):
        i0, n = C.c_int64(), C.c_int64()
        self.ctx.check(lib().lpk_batch_round_extent(self.h, rnd, unit, C.byref(i0), C.byref(n)))
        return i0.value, n.value

    def run(self, rnd: int):
        self.ctx.check(lib().lpk_batch_run(self.h, rnd))

    def output(self, unit: int) -> np.ndarray:
        """Copy of unit's output of the last round (complex64)."""
        buf = np.zeros(self._caps[unit], dtype=np.complex64)
        self.ctx.check(lib().lpk_batch_copy_out(self.h, unit, buf.ctypes.data_as(_CF), buf.size))
        return buf

    def config(self):
        v, b, m = C.c_int32(), C.c_int32(), C.c_int32()
        self.ctx.check(lib().lpk_batch_get_config(self.h, C.byref(v), C.byref(b), C.byref(m)))
        return v.value, b.value, m.value

    def set_config(self, variant: int, blocks_per_sm: int = 0):
        self.ctx.check(lib().lpk_batch_set_config(self.h, variant, blocks_per_sm))

    def autotune(self, rnd: int = 0, reps: int = 2):
        nv = lib().lpk_split_variant_count()
        tab = np.zeros(2 * nv, dtype=np.float64)
        self.ctx.check(lib().lpk_batch_autotune(self.h, rnd, reps, tab.ctypes.data_as(_D)))
        return tab.reshape(nv, 2)

    def render(self):
        """Every round through lpk_batch_render (double-buffered copies to
        pinned staging); returns one complex64 array per unit."""
        outs = [[] for _ in range(self.n_units)]
        err: list = []

        def _sink(_user, u, ptr, n):
            try:
                arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(2 * n,)).copy()
                outs[u].append(arr.view(np.complex64))
                return 0
            except BaseException as e:
                err.append(e)
                return -1

        cb = UNIT_SINK_FN(_sink)
        code = lib().lpk_batch_render(self.h, cb, None)
        if err:
            raise err[0]
        self.ctx.check(code)
        return [np.concatenate(o) if o else np.zeros(0, np.complex64) for o in outs]


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


class Mlp:
    """lpk_mlp: the warm-start network of the converged emission solve."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        h = _VP()
        ctx.check(lib().lpk_mlp_create(ctx.h, seed & 0xFFFFFFFFFFFFFFFF, C.byref(h)))
        self.h = h
        ctx.adopt(self)

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().lpk_mlp_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def __del__(self):
        self.close()

    def params(self):
        p = np.zeros(MLP_N_PARAMS, np.float32)
        nrm = np.zeros(MLP_N_NORM, np.float32)
        self.ctx.check(lib().lpk_mlp_get_params(self.h, _fp(p), _fp(nrm)))
        return p, nrm

    def set_params(self, p, norm=None):
        p = np.ascontiguousarray(p, np.float32)
        nrm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        self.ctx.check(lib().lpk_mlp_set_params(self.h, _fp(p), None if nrm is None else _fp(nrm)))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros(len(x), np.float32)
        self.ctx.check(lib().lpk_mlp_forward(self.h, _fp(x), len(x), _fp(y)))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(MLP_N_PARAMS, np.float32)
        loss = C.c_double()
        self.ctx.check(lib().lpk_mlp_loss_grad(self.h, _fp(x), _fp(t), len(x), C.byref(loss), _fp(g)))
        return loss.value, g

    def fit(self, txs, orbits, rx_ecef, epoch, t0, t1, n_train=1 << 21, steps=2000, batch=4096, lr=3e-3, seed=1):
        """Train the scene's surrogate: txs (uploaded indices) with their
        circular orbits (KeplerOrbit each), rx_ecef (n_rx, 3) receivers,
        reception times in [t0, t1). Returns the per-step batch loss."""
        tx = np.ascontiguousarray(np.asarray(txs, np.int32))
        orb = (KeplerOrbit * len(orbits))(*orbits)
        rx = np.ascontiguousarray(np.asarray(rx_ecef, np.float64).reshape(-1, 3))
        curve = np.zeros(steps, np.float32)
        self.ctx.check(lib().lpk_mlp_fit(self.h, tx.ctypes.data_as(_I32), orb, len(tx), dptr(rx), len(rx), epoch, t0,
                                         t1, n_train, steps, batch, lr, seed & 0xFFFFFFFFFFFFFFFF, _fp(curve)))
        return curve

    def set_orbits(self, txs, orbits):
        tx = np.ascontiguousarray(np.asarray(txs, np.int32))
        orb = (KeplerOrbit * len(orbits))(*orbits)
        self.ctx.check(lib().lpk_mlp_set_orbits(self.h, tx.ctypes.data_as(_I32), orb, len(tx)))

    def features(self, tx, rx_ecef, epoch, t_rel_utc):
        t = np.ascontiguousarray(t_rel_utc, np.float64)
        rx = np.ascontiguousarray(rx_ecef, np.float64)
        f = np.zeros((len(t), MLP_N_FEATURES), np.float32)
        self.ctx.check(lib().lpk_mlp_features(self.h, tx, dptr(rx), epoch, dptr(t), len(t), _fp(f)))
        return f


def solve_converged(ctx: Context, tx, rx_ecef, epoch, t_rel_utc, tol=1e-13, max_iter=12,
                    scheme=LPK_ITER_NEWTON, start=LPK_START_LAG, mlp: "Mlp | None" = None):
    """Converged emission solve: (t_emit, iterations, |start - converged| in s)."""
    t = np.ascontiguousarray(t_rel_utc, np.float64)
    rx = np.ascontiguousarray(rx_ecef, np.float64)
    te = np.zeros(len(t))
    it = np.zeros(len(t), np.int32)
    err = np.zeros(len(t), np.float32)
    ctx.check(lib().lpk_solve_converged(ctx.h, tx, dptr(rx), epoch, dptr(t), len(t), tol, max_iter, scheme, start,
                                        mlp.h if mlp is not None else None, dptr(te),
                                        it.ctypes.data_as(_I32), _fp(err)))
    return te, it, err


def solve_converged_scene(ctx: Context, tx, rx_idx, rx_ecef, epoch, t_rel_utc, tol=1e-13, max_iter=12,
                          scheme=LPK_ITER_NEWTON, start=LPK_START_LAG, mlp: "Mlp | None" = None):
    """Converged emission solve over (transmitter, receiver) pairs:
    (t_emit, iterations, |start - converged| in s, device ms)."""
    t = np.ascontiguousarray(t_rel_utc, np.float64)
    txa = np.ascontiguousarray(np.asarray(tx, np.int32))
    rxa = np.ascontiguousarray(np.asarray(rx_idx, np.int32))
    rx = np.ascontiguousarray(np.asarray(rx_ecef, np.float64).reshape(-1, 3))
    te = np.zeros(len(t))
    it = np.zeros(len(t), np.int32)
    err = np.zeros(len(t), np.float32)
    ms = C.c_double()
    ctx.check(lib().lpk_solve_converged_scene(ctx.h, txa.ctypes.data_as(_I32), rxa.ctypes.data_as(_I32), dptr(rx),
                                              len(rx), epoch, dptr(t), len(t), tol, max_iter, scheme, start,
                                              mlp.h if mlp is not None else None, dptr(te), it.ctypes.data_as(_I32),
                                              _fp(err), C.byref(ms)))
    return te, it, err, ms.value


def scene_orbits(scene):
    """(transmitter indices, KeplerOrbit per index) of a scene's transmitters
    on circular Keplerian orbits: the inputs of the scene's surrogate."""
    txs, orbits = [], []
    for i, t in enumerate(scene.transmitters):
        if t.trajectory.kind != "circular_keplerian":
            continue
        p = t.trajectory.params
        txs.append(i)
        orbits.append(KeplerOrbit(p["semi_major_axis_m"], p["inclination_deg"], p["raan_deg"],
                                  p["true_anomaly_deg_at_epoch"], p.get("epoch_unix", scene.epoch_unix)))
    return txs, orbits
