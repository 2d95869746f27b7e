"""Scene orchestration on the B200 backend: the reference's pipeline API.

Mirrors src/pipeline.rs: `run_scene` (:443), `run_scene_to_dir` (:494),
`render_window` (:709), `export_truth` (:548) and the output layout of
src/output/mod.rs (raw complex64 + JSON sidecar). The per-chunk work runs in
liblipika_cuda.so; this module only prepares the scene description and
collects the chunks.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import config as cfgmod
from . import native as N
from . import scene_abi as A

DEFAULT_CHUNK_SAMPLES = 1 << 20          # src/pipeline.rs:367
DEFAULT_WINDOW_CHUNK_SAMPLES = 1 << 16   # src/pipeline.rs:637
DEFAULT_SIGNAL_EPOCH_UNIX = 0.0          # src/pipeline.rs:139
SPEED_OF_LIGHT = 299_792_458.0


@dataclass
class ObserverOutput:
    """One band's IQ and its metadata (src/output/mod.rs:21-33)."""
    name: str
    epoch_unix: float
    sample_rate_hz: float
    lo_carrier_hz: float
    iq: np.ndarray
    descriptor: dict

    def write_raw_with_sidecar(self, directory: str):  # output/mod.rs:39-50
        os.makedirs(directory, exist_ok=True)
        self.iq.astype(np.complex64).tofile(os.path.join(directory, f"{self.name}.iq.c64"))
        write_sidecar(directory, self.name, self.epoch_unix, self.sample_rate_hz, self.lo_carrier_hz,
                      len(self.iq), self.descriptor)


@dataclass
class OutputManifest:  # src/pipeline.rs:431-437
    name: str
    path: str
    n_samples: int
    descriptor: dict


@dataclass
class WindowOptions:  # src/pipeline.rs:623-643
    seed: int = 0
    chunk_samples: int = DEFAULT_WINDOW_CHUNK_SAMPLES
    n_threads: int = 1


@dataclass
class WindowSummary:  # src/pipeline.rs:646-669
    n_samples_window: int
    n_samples_emitted: int
    stopped_early: bool
    contributing_transmitters: list = field(default_factory=list)
    visible_transmitters: list = field(default_factory=list)


def sidecar_json(name, epoch_unix, fs, lo, n, descriptor) -> dict:  # output/mod.rs:56-74
    return {
        "name": name, "epoch_unix": epoch_unix, "sample_rate_hz": fs, "lo_carrier_hz": lo,
        "n_samples": n, "format": "raw complex64 little-endian (interleaved f32 re, f32 im)",
        "numpy_load": "np.fromfile(path, dtype=np.complex64)", "descriptor": descriptor,
    }


def write_sidecar(directory, name, epoch_unix, fs, lo, n, descriptor):
    with open(os.path.join(directory, f"{name}.iq.json"), "w") as f:
        json.dump(sidecar_json(name, epoch_unix, fs, lo, n, descriptor), f, indent=2)


def _tx_descriptor(t: cfgmod.Transmitter) -> dict:  # src/pipeline.rs:1083-1097
    d = {"name": t.name, "kind": t.kind, "carrier_hz": t.carrier_hz, "tx_power_dbw": t.tx_power_dbw,
         "bandwidth_hz": t.effective_bandwidth_hz(), "trajectory_kind": t.trajectory.kind}
    if t.kind == "ca_code":
        d["prn"] = t.params["prn"]
        d["nav"] = t.params["nav"]
    return d


def _scene_json(scene: cfgmod.Scene) -> dict:
    import dataclasses
    return dataclasses.asdict(scene)


class Prepared:
    """A scene prepared on a context (prepare, src/pipeline.rs:801-819)."""

    def __init__(self, scene: cfgmod.Scene, ctx: Optional[N.Context] = None,
                 time_base: int = A.LPK_TIME_BASE_SCENE,
                 default_signal_epoch_unix: float = DEFAULT_SIGNAL_EPOCH_UNIX, device_tables: bool = False):
        """device_tables: build the circular Keplerian trajectory tables on the
        GPU (lpk_kepler_tables) instead of the host."""
        self.scene = scene
        self.ctx = ctx or N.Context(0)
        self.cs = cfgmod.to_c(scene, time_base, default_signal_epoch_unix)
        self.cs.cfg.flags = A.LPK_SCENE_DEVICE_TABLES if device_tables else 0
        h = C.c_void_p()
        N.check(N.lib().lpk_scene_prepare(self.ctx.h, C.byref(self.cs.cfg), C.byref(h)), self.ctx.h)
        self.h = h
        self.ctx.adopt(self)

    def close(self):
        if getattr(self, "h", None):
            try:
                N.lib().lpk_scene_free(self.h)
            except Exception:  # interpreter shutdown
                pass
            self.h = None

    def __del__(self):
        self.close()

    def work(self):
        L = N.lib()
        out = []
        for w in range(L.lpk_scene_n_work(self.h)):
            r, b = C.c_int32(), C.c_int32()
            N.check(L.lpk_scene_work(self.h, w, C.byref(r), C.byref(b)))
            out.append((r.value, b.value))
        return out

    def n_samples(self, r, b) -> int:
        return N.lib().lpk_scene_band_samples(self.h, r, b)

    def active(self, r, b):
        buf = (C.c_int32 * 256)()
        k = N.lib().lpk_scene_band_active(self.h, r, b, buf, 256)
        return [buf[i] for i in range(min(k, 256))]

    def band_desc(self, r, b, seed, work_idx) -> N.BandDesc:
        d = N.BandDesc()
        N.check(N.lib().lpk_scene_band_desc(self.h, r, b, seed & 0xFFFFFFFFFFFFFFFF, work_idx, C.byref(d)))
        return d

    def generate_band(self, r: int, b: int, seed: int, work_idx: int, chunk_samples: int,
                      sink: Callable[[np.ndarray], bool], noise: bool = True,
                      device_clock: bool = False, split: bool = False) -> N.BandResult:
        """generate_band (src/pipeline.rs:836-1019); `sink(chunk)` returns True to stop.

        device_clock=True draws the receiver's white-FM walk on the GPU
        (counter-based, moment-matched) instead of the host stream."""
        err: list = []

        def _sink(_user, ptr, n):
            try:
                arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(2 * n,)).copy()
                return 1 if sink(arr.view(np.complex64)) else 0
            except BaseException as e:  # propagate after the native loop returns
                err.append(e)
                return -1

        cb = N.SINK_FN(_sink)
        res = N.BandResult()
        flags = (N.LPK_NOISE_ON if noise else N.LPK_NOISE_OFF) | (N.LPK_GEN_DEVICE_CLOCK if device_clock else 0) \
            | (N.LPK_GEN_SPLIT if split else 0)
        code = N.lib().lpk_generate_band(self.h, r, b, seed & 0xFFFFFFFFFFFFFFFF, work_idx, max(1, chunk_samples),
                                         flags, cb, None, C.byref(res))
        if err:
            raise err[0]
        N.check(code, self.ctx.h)
        return res

    def generate_scene(self, seed: int, round_s: float, sink: Callable[[int, np.ndarray], bool],
                       noise: bool = True, device_clock: bool = True, split: bool = True,
                       autotune: bool = False) -> None:
        """Every work unit at once through the batched fan-out
        (lpk_generate_scene): `sink(work_idx, chunk)` receives each unit's
        chunks in order and returns True to stop that unit."""
        err: list = []

        def _sink(_user, w, ptr, n):
            try:
                arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(2 * n,)).copy()
                return 1 if sink(int(w), arr.view(np.complex64)) else 0
            except BaseException as e:
                err.append(e)
                return -1

        cb = N.UNIT_SINK_FN(_sink)
        flags = (N.LPK_NOISE_ON if noise else N.LPK_NOISE_OFF) | (N.LPK_GEN_DEVICE_CLOCK if device_clock else 0) \
            | (N.LPK_GEN_SPLIT if split else 0) | (N.LPK_GEN_AUTOTUNE if autotune else 0)
        code = N.lib().lpk_generate_scene(self.h, seed & 0xFFFFFFFFFFFFFFFF, float(round_s), flags, cb, None)
        if err:
            raise err[0]
        N.check(code, self.ctx.h)

    def band_meta(self, r: int, b: int, contributing_idx) -> dict:
        rx = self.scene.receivers[r]
        band = rx.bands[b]
        noise = band.noise_power_w if band.noise_power_w is not None else \
            1.380649e-23 * band.noise_temperature_k * band.sample_rate_hz
        return {  # src/pipeline.rs:992-1005
            "receiver": rx.name, "band_id": band.band_id, "duration_s": self.scene.duration_s,
            "band": {"lo_carrier_hz": band.lo_carrier_hz, "sample_rate_hz": band.sample_rate_hz,
                     "bandwidth_hz": band.effective_bandwidth_hz(),
                     "noise_temperature_k": band.noise_temperature_k, "noise_power_w": noise},
            "contributing_transmitters": [_tx_descriptor(self.scene.transmitters[i]) for i in contributing_idx],
            "scene_config": _scene_json(self.scene),
        }


def run_scene(scene: cfgmod.Scene, rng_seed_base: int, ctx: Optional[N.Context] = None,
              chunk_samples: int = DEFAULT_CHUNK_SAMPLES, noise: bool = True) -> list[ObserverOutput]:
    """In-memory render of every (receiver, band) (src/pipeline.rs:443-485)."""
    p = Prepared(scene, ctx)
    outs = []
    for work_idx, (r, b) in enumerate(p.work()):
        rx = scene.receivers[r]
        band = rx.bands[b]
        chunks: list = []
        p.generate_band(r, b, rng_seed_base, work_idx, chunk_samples, lambda c: chunks.append(c) and False,
                        noise)
        iq = np.concatenate(chunks) if chunks else np.zeros(0, np.complex64)
        outs.append(ObserverOutput(f"{rx.name}__{band.band_id}", scene.epoch_unix, band.sample_rate_hz,
                                   band.lo_carrier_hz, iq, p.band_meta(r, b, p.active(r, b))))
    p.close()
    return outs


def run_scene_to_dir(scene: cfgmod.Scene, rng_seed_base: int, directory: str,
                     chunk_samples: int = DEFAULT_CHUNK_SAMPLES, n_threads: int = 0,
                     ctx: Optional[N.Context] = None, noise: bool = True, device_clock: bool = False,
                     round_s: float = 4.0) -> list[OutputManifest]:
    """Stream each band to <dir>/<rx>__<band>.iq.c64 + .iq.json (src/pipeline.rs:494-536).

    `n_threads` is accepted for signature parity; the fan-out runs on the GPU.
    With device_clock=True every band is rendered by one batch
    (lpk_generate_scene_to_files: clock walks on the GPU, split fan-out,
    rounds of round_s seconds written while the next round renders);
    otherwise band by band with the host clock stream."""
    os.makedirs(directory, exist_ok=True)
    p = Prepared(scene, ctx)
    out = []
    if device_clock:
        names = [f"{scene.receivers[r].name}__{scene.receivers[r].bands[b].band_id}" for (r, b) in p.work()]
        paths = [os.path.join(directory, f"{nm}.iq.c64") for nm in names]
        arr = (C.c_char_p * len(paths))(*[x.encode() for x in paths])
        flags = (N.LPK_NOISE_ON if noise else N.LPK_NOISE_OFF) | N.LPK_GEN_DEVICE_CLOCK | N.LPK_GEN_SPLIT
        N.check(N.lib().lpk_generate_scene_to_files(p.h, rng_seed_base & 0xFFFFFFFFFFFFFFFF, float(round_s), flags,
                                                     arr), p.ctx.h)
        for (r, b), nm, path in zip(p.work(), names, paths):
            band = scene.receivers[r].bands[b]
            n = p.n_samples(r, b)
            desc = p.band_meta(r, b, p.active(r, b))
            write_sidecar(directory, nm, scene.epoch_unix, band.sample_rate_hz, band.lo_carrier_hz, n, desc)
            out.append(OutputManifest(nm, path, n, desc))
        p.close()
        return out
    for work_idx, (r, b) in enumerate(p.work()):
        rx = scene.receivers[r]
        band = rx.bands[b]
        name = f"{rx.name}__{band.band_id}"
        path = os.path.join(directory, f"{name}.iq.c64")
        res = N.BandResult()
        N.check(N.lib().lpk_generate_band_to_file(p.h, r, b, rng_seed_base & 0xFFFFFFFFFFFFFFFF, work_idx,
                                                  max(1, chunk_samples),
                                                  N.LPK_NOISE_ON if noise else N.LPK_NOISE_OFF,
                                                  path.encode(), C.byref(res)), p.ctx.h)
        desc = p.band_meta(r, b, p.active(r, b))
        write_sidecar(directory, name, scene.epoch_unix, band.sample_rate_hz, band.lo_carrier_hz,
                      int(res.n_samples), desc)
        out.append(OutputManifest(name, path, int(res.n_samples), desc))
    p.close()
    return out


def render_window(sky: cfgmod.Sky, receiver: cfgmod.Receiver, band: cfgmod.Band, start_unix: float,
                  duration_s: float, options: WindowOptions, sink: Callable[[np.ndarray], bool],
                  ctx: Optional[N.Context] = None) -> WindowSummary:
    """One receiver, one band, one absolute-time window of a sky (src/pipeline.rs:709-794).

    `sink(chunk)` returns True to stop the render after that chunk."""
    if not math.isfinite(start_unix):
        raise ValueError(f"window start_unix must be finite, got {start_unix}")
    if not (duration_s >= 0.0) or not math.isfinite(duration_s):
        raise ValueError(f"window duration_s must be finite and non-negative, got {duration_s}")
    if not (band.sample_rate_hz > 0.0) or not math.isfinite(band.sample_rate_hz):
        raise ValueError(f"band sample_rate_hz must be positive, got {band.sample_rate_hz}")
    rx = cfgmod.replace(receiver, bands=[band])
    scene = cfgmod.Scene(start_unix, duration_s, list(sky.transmitters), [rx], sky.gps_utc_offset_s)
    p = Prepared(scene, ctx, A.LPK_TIME_BASE_ABSOLUTE, DEFAULT_SIGNAL_EPOCH_UNIX)
    res = p.generate_band(0, 0, options.seed, 0, max(1, options.chunk_samples), sink)
    active = p.active(0, 0)
    names = [sky.transmitters[i].name for i in active]
    visible = [nm for k, nm in enumerate(names) if res.unoccluded[k]]
    p.close()
    return WindowSummary(round(band.sample_rate_hz * duration_s), int(res.n_samples), bool(res.stopped_early),
                         names, visible)


def export_truth(scene: cfgmod.Scene, directory: str, truth_hz: float, ctx: Optional[N.Context] = None):
    """Geometric truth per (receiver, transmitter) on a coarse grid (src/pipeline.rs:548-612)."""
    if truth_hz <= 0.0:
        return
    os.makedirs(directory, exist_ok=True)
    p = Prepared(scene, ctx)
    epoch, dur = scene.epoch_unix, scene.duration_s
    ng = max(round(dur * truth_hz), 1) + 1
    dt = 1.0 / truth_hz
    t_rel = np.arange(ng, dtype=np.float64) * dt
    L = N.lib()
    for r, rx in enumerate(scene.receivers):
        b = cfgmod.Band("truth", 0.0, 1.0)
        pos = np.zeros(3)
        desc = p.band_desc(r, 0, 0, 0)
        pos[:] = list(desc.rx_ecef)
        obs = np.ascontiguousarray(np.repeat(pos[:, None], ng, axis=1))
        txs = []
        for i, t in enumerate(scene.transmitters):
            te = np.zeros(ng)
            rg = np.zeros(ng)
            N.check(L.lpk_solve_emission_times(p.ctx.h, i, N.dptr(obs), N.dptr(t_rel), ng, epoch, 4,
                                               N.dptr(te), N.dptr(rg)), p.ctx.h)
            rr = np.gradient(rg, dt) if ng >= 2 else np.zeros(ng)
            if ng >= 2:
                rr[0] = (rg[1] - rg[0]) / dt
                rr[-1] = (rg[-1] - rg[-2]) / dt
            d = _tx_descriptor(t)
            d.update(range_m=rg.tolist(), delay_s=(rg / SPEED_OF_LIGHT).tolist(), range_rate_m_s=rr.tolist())
            txs.append(d)
        del b
        with open(os.path.join(directory, f"{rx.name}__truth.json"), "w") as f:
            json.dump({"receiver": rx.name, "epoch_unix": epoch, "duration_s": dur, "grid_hz": truth_hz,
                       "t_utc": (epoch + t_rel).tolist(), "transmitters": txs}, f)
    p.close()
