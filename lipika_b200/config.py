"""Scene configuration: the reference's TOML schema in Python.

Mirrors src/config/mod.rs:52-467 (SceneConfig, SkyConfig, TransmitterConfig,
ReceiverConfig, ReceiverBandConfig, FrontendConfig, TrajectoryConfig,
NodeClockSpec) including its defaults, and lowers a scene to the flat C
description of include/lipika_scene.h (`to_c`).
"""
from __future__ import annotations

import copy
import ctypes as C
import dataclasses
import tomllib
from dataclasses import dataclass, field
from typing import Any, Optional

from . import scene_abi as A

CA_CHIP_RATE_HZ = 1_023_000.0  # src/signal/ca_code.rs:23


class ConfigError(ValueError):
    """A scene that the reference would reject while parsing or preparing it."""


@dataclass
class Trajectory:
    kind: str
    params: dict

    def kind_name(self) -> str:  # src/config/mod.rs:451-459
        return self.kind


@dataclass
class Gate:
    period_s: float
    bursts: list  # [(offset_s, duration_s)]
    epoch_unix: float = 0.0


@dataclass
class Transmitter:
    name: str
    carrier_hz: float
    kind: str
    params: dict
    trajectory: Trajectory
    tx_power_dbw: float = 0.0
    bandwidth_hz: Optional[float] = None
    signal_epoch_unix: Optional[float] = None
    gate: Optional[Gate] = None

    def default_bandwidth_hz(self) -> float:  # src/config/mod.rs:260-268
        if self.kind == "cw":
            return 0.0
        if self.kind in ("bpsk", "ook"):
            return 2.0 * self.params["bit_rate_bps"]
        if self.kind == "qam16":
            return 2.0 * self.params["symbol_rate_baud"]
        return 2.0 * CA_CHIP_RATE_HZ

    def effective_bandwidth_hz(self) -> float:  # src/config/mod.rs:191-193
        return self.bandwidth_hz if self.bandwidth_hz is not None else self.default_bandwidth_hz()


@dataclass
class Clock:
    allan_deviation_1s: float = 0.0
    flicker_floor: float = 0.0
    frequency_offset_y0: float = 0.0
    initial_time_offset_s: float = 0.0


@dataclass
class Frontend:
    antenna: Optional[dict] = None  # peak_dbi, horizon_dbi, fb_db, cutoff_deg?
    gain_db: Optional[float] = None
    iip3_dbm: Optional[float] = None
    adc_bits: Optional[int] = None
    adc_full_scale_v: Optional[float] = None


@dataclass
class Band:
    band_id: str
    lo_carrier_hz: float
    sample_rate_hz: float
    noise_temperature_k: float = 290.0
    noise_power_w: Optional[float] = None
    bandwidth_hz: Optional[float] = None
    frontend: Optional[Frontend] = None

    def effective_bandwidth_hz(self) -> float:  # src/config/mod.rs:420-422
        return self.bandwidth_hz if self.bandwidth_hz is not None else self.sample_rate_hz


@dataclass
class Receiver:
    name: str
    trajectory: Trajectory
    clock: Clock = field(default_factory=Clock)
    bands: list = field(default_factory=list)


@dataclass
class Scene:
    epoch_unix: float
    duration_s: float
    transmitters: list = field(default_factory=list)
    receivers: list = field(default_factory=list)
    gps_utc_offset_s: float = 18.0

    def clone(self) -> "Scene":
        return copy.deepcopy(self)


@dataclass
class Sky:
    transmitters: list = field(default_factory=list)
    gps_utc_offset_s: float = 18.0


_TRAJ_FIELDS = {
    "stationary_geodetic": ("lat_deg", "lon_deg", "h_m"),
    "stationary_ecef": ("x_m", "y_m", "z_m"),
    "circular_keplerian": ("semi_major_axis_m", "inclination_deg", "raan_deg",
                           "true_anomaly_deg_at_epoch", "epoch_unix"),
    "tle": ("line1", "line2"),
    "rinex_nav": ("file", "prn"),
}
_KIND_FIELDS = {
    "cw": ("baseband_offset_hz",),
    "bpsk": ("bit_rate_bps", "payload_bits", "payload_seed", "sync_word"),
    "ook": ("bit_rate_bps", "payload_bits", "payload_seed", "sync_word"),
    "qam16": ("symbol_rate_baud", "payload_symbols", "payload_seed", "sync_word"),
    "ca_code": ("prn", "epoch_unix"),
}


def _need(d: dict, key: str, ctx: str):
    if key not in d:
        raise ConfigError(f"{ctx}: missing field `{key}`")
    return d[key]


def _traj(d: dict, ctx: str) -> Trajectory:
    kind = _need(d, "kind", ctx)
    if kind not in _TRAJ_FIELDS:
        raise ConfigError(f"{ctx}: unknown trajectory kind `{kind}`")
    params = {k: _need(d, k, ctx) for k in _TRAJ_FIELDS[kind]}
    return Trajectory(kind, params)


def _transmitter(d: dict) -> Transmitter:
    name = _need(d, "name", "transmitter")
    ctx = f"transmitter '{name}'"
    kind = _need(d, "kind", ctx)
    if kind not in _KIND_FIELDS:
        raise ConfigError(f"{ctx}: unknown kind `{kind}`")
    params = {k: _need(d, k, ctx) for k in _KIND_FIELDS[kind]}
    if kind == "ca_code":
        params["nav"] = d.get("nav", "dummy")  # NavMode default (src/config/mod.rs:227-237)
        params["nav_seed"] = int(d.get("nav_seed", 0))
        if params["nav"] not in ("off", "dummy", "full"):
            raise ConfigError(f"{ctx}: unknown nav mode `{params['nav']}`")
    gate = None
    if "gate" in d:
        g = d["gate"]
        gate = Gate(period_s=float(_need(g, "period_s", ctx)),
                    bursts=[(float(b["offset_s"]), float(b["duration_s"])) for b in _need(g, "bursts", ctx)],
                    epoch_unix=float(g.get("epoch_unix", 0.0)))
    return Transmitter(
        name=name, carrier_hz=float(_need(d, "carrier_hz", ctx)), kind=kind, params=params,
        trajectory=_traj(_need(d, "trajectory", ctx), ctx),
        tx_power_dbw=float(d.get("tx_power_dbw", 0.0)),
        bandwidth_hz=None if d.get("bandwidth_hz") is None else float(d["bandwidth_hz"]),
        signal_epoch_unix=None if d.get("signal_epoch_unix") is None else float(d["signal_epoch_unix"]),
        gate=gate,
    )


def _frontend(d: Optional[dict]) -> Optional[Frontend]:
    if d is None:
        return None
    fe = Frontend()
    if d.get("antenna") is not None:
        a = d["antenna"]
        fe.antenna = {"peak_dbi": float(a["peak_dbi"]), "horizon_dbi": float(a["horizon_dbi"]),
                      "fb_db": float(a["fb_db"]), "cutoff_deg": a.get("cutoff_deg")}
    fe.gain_db = d.get("gain_db")
    if d.get("nonlinearity") is not None:
        fe.iip3_dbm = float(d["nonlinearity"]["iip3_dbm"])
    if d.get("adc") is not None:
        fe.adc_bits = int(d["adc"]["bits"])
        fe.adc_full_scale_v = float(d["adc"]["full_scale_v"])
    return fe


def _receiver(d: dict) -> Receiver:
    name = _need(d, "name", "receiver")
    ctx = f"receiver '{name}'"
    c = d.get("clock", {})
    clock = Clock(float(c.get("allan_deviation_1s", 0.0)), float(c.get("flicker_floor", 0.0)),
                  float(c.get("frequency_offset_y0", 0.0)), float(c.get("initial_time_offset_s", 0.0)))
    bands = []
    for b in d.get("band", []):
        bands.append(Band(
            band_id=_need(b, "band_id", ctx), lo_carrier_hz=float(_need(b, "lo_carrier_hz", ctx)),
            sample_rate_hz=float(_need(b, "sample_rate_hz", ctx)),
            noise_temperature_k=float(b.get("noise_temperature_k", 290.0)),
            noise_power_w=None if b.get("noise_power_w") is None else float(b["noise_power_w"]),
            bandwidth_hz=None if b.get("bandwidth_hz") is None else float(b["bandwidth_hz"]),
            frontend=_frontend(b.get("frontend"))))
    return Receiver(name=name, trajectory=_traj(_need(d, "trajectory", ctx), ctx), clock=clock, bands=bands)


def scene_from_dict(doc: dict) -> Scene:
    meta = _need(doc, "scene", "scene file")
    return Scene(
        epoch_unix=float(_need(meta, "epoch_unix", "[scene]")),
        duration_s=float(_need(meta, "duration_s", "[scene]")),
        gps_utc_offset_s=float(meta.get("gps_utc_offset_s", 18.0)),
        transmitters=[_transmitter(t) for t in doc.get("transmitter", [])],
        receivers=[_receiver(r) for r in doc.get("receiver", [])],
    )


def scene_from_toml_str(text: str) -> Scene:
    """SceneConfig parsing (src/config/mod.rs:462-466)."""
    return scene_from_dict(tomllib.loads(text))


def scene_from_toml_file(path) -> Scene:
    with open(path, "rb") as f:
        return scene_from_dict(tomllib.load(f))


def sky_from_toml_str(text: str) -> Sky:
    """SkyConfig::from_toml_str (src/config/mod.rs:176-178)."""
    doc = tomllib.loads(text)
    extra = set(doc) - {"transmitter", "gps_utc_offset_s"}
    if extra:
        raise ConfigError(f"sky: unknown field(s) {sorted(extra)}")
    return Sky([_transmitter(t) for t in doc.get("transmitter", [])],
               float(doc.get("gps_utc_offset_s", 18.0)))


# ---------------------------------------------------------------------------
# Lowering to the C description.
# ---------------------------------------------------------------------------
class CScene:
    """A `lpk_scene_cfg` plus every array it points to (kept alive here)."""

    def __init__(self, scene: Scene, time_base: int = A.LPK_TIME_BASE_SCENE,
                 default_signal_epoch_unix: float = 0.0):
        self._keep: list[Any] = []
        ntx = len(scene.transmitters)
        txs = (A.TransmitterCfg * max(ntx, 1))()
        for i, t in enumerate(scene.transmitters):
            self._fill_tx(txs[i], t)
        nrx = len(scene.receivers)
        rxs = (A.ReceiverCfg * max(nrx, 1))()
        for i, r in enumerate(scene.receivers):
            self._fill_rx(rxs[i], r)
        self._keep += [txs, rxs]
        self.cfg = A.SceneCfg(
            epoch_unix=scene.epoch_unix, duration_s=scene.duration_s,
            gps_utc_offset_s=scene.gps_utc_offset_s,
            default_signal_epoch_unix=default_signal_epoch_unix, time_base=time_base,
            n_transmitters=ntx, transmitters=txs, n_receivers=nrx, receivers=rxs)

    @staticmethod
    def _traj(c: A.TrajectoryCfg, t: Trajectory):
        kinds = {"stationary_geodetic": A.LPK_TRAJ_STATIONARY_GEODETIC,
                 "stationary_ecef": A.LPK_TRAJ_STATIONARY_ECEF,
                 "circular_keplerian": A.LPK_TRAJ_CIRCULAR_KEPLERIAN,
                 "tle": A.LPK_TRAJ_TLE, "rinex_nav": A.LPK_TRAJ_RINEX_NAV}
        c.kind = kinds[t.kind]
        for k, v in t.params.items():
            if k in ("line1", "line2", "file", "prn"):
                continue
            setattr(c, k, float(v))

    def _fill_tx(self, c: A.TransmitterCfg, t: Transmitter):
        kinds = {"cw": A.LPK_SIG_CW, "bpsk": A.LPK_SIG_BPSK, "ook": A.LPK_SIG_OOK,
                 "qam16": A.LPK_SIG_QAM16, "ca_code": A.LPK_SIG_CA_CODE}
        c.carrier_hz = t.carrier_hz
        c.tx_power_dbw = t.tx_power_dbw
        c.kind = kinds[t.kind]
        c.has_bandwidth = int(t.bandwidth_hz is not None)
        c.bandwidth_hz = t.bandwidth_hz or 0.0
        self._traj(c.trajectory, t.trajectory)
        c.has_signal_epoch = int(t.signal_epoch_unix is not None)
        c.signal_epoch_unix = t.signal_epoch_unix or 0.0
        if t.gate is not None:
            c.has_gate = 1
            c.gate_period_s = t.gate.period_s
            c.gate_epoch_unix = t.gate.epoch_unix
            flat = [v for b in t.gate.bursts for v in b]
            arr = (C.c_double * max(len(flat), 1))(*flat)
            self._keep.append(arr)
            c.gate_n_bursts = len(t.gate.bursts)
            c.gate_bursts = C.cast(arr, C.POINTER(C.c_double))
        p = t.params
        if t.kind == "cw":
            c.baseband_offset_hz = float(p["baseband_offset_hz"])
        elif t.kind in ("bpsk", "ook", "qam16"):
            c.rate_hz = float(p["bit_rate_bps"] if t.kind != "qam16" else p["symbol_rate_baud"])
            c.payload_n = int(p["payload_bits"] if t.kind != "qam16" else p["payload_symbols"])
            c.payload_seed = int(p["payload_seed"]) & 0xFFFFFFFFFFFFFFFF
            sw = [int(v) for v in p["sync_word"]]
            if any(v < -128 or v > 127 for v in sw):
                raise ConfigError("sync_word entries out of range")
            arr = (C.c_int8 * max(len(sw), 1))(*sw)
            self._keep.append(arr)
            c.sync_n = len(sw)
            c.sync_word = C.cast(arr, C.POINTER(C.c_int8))
        else:
            c.prn = int(p["prn"])
            c.ca_epoch_unix = float(p["epoch_unix"])
            c.nav = {"off": A.LPK_NAV_OFF, "dummy": A.LPK_NAV_DUMMY, "full": A.LPK_NAV_FULL}[p["nav"]]
            c.nav_seed = int(p["nav_seed"]) & 0xFFFFFFFFFFFFFFFF

    def _fill_rx(self, c: A.ReceiverCfg, r: Receiver):
        self._traj(c.trajectory, r.trajectory)
        c.clock = A.ClockCfg(r.clock.allan_deviation_1s, r.clock.flicker_floor,
                             r.clock.frequency_offset_y0, r.clock.initial_time_offset_s)
        bands = (A.BandCfg * max(len(r.bands), 1))()
        for i, b in enumerate(r.bands):
            bc = bands[i]
            bc.lo_carrier_hz = b.lo_carrier_hz
            bc.sample_rate_hz = b.sample_rate_hz
            bc.noise_temperature_k = b.noise_temperature_k
            bc.has_noise_power = int(b.noise_power_w is not None)
            bc.noise_power_w = b.noise_power_w or 0.0
            bc.has_bandwidth = int(b.bandwidth_hz is not None)
            bc.bandwidth_hz = b.bandwidth_hz or 0.0
            fe = b.frontend
            if fe is not None:
                bc.has_frontend = 1
                f = bc.frontend
                if fe.antenna is not None:
                    f.has_antenna = 1
                    f.peak_dbi = fe.antenna["peak_dbi"]
                    f.horizon_dbi = fe.antenna["horizon_dbi"]
                    f.fb_db = fe.antenna["fb_db"]
                    if fe.antenna.get("cutoff_deg") is not None:
                        f.has_cutoff = 1
                        f.cutoff_deg = float(fe.antenna["cutoff_deg"])
                if fe.gain_db is not None:
                    f.has_gain = 1
                    f.gain_db = float(fe.gain_db)
                if fe.iip3_dbm is not None:
                    f.has_nonlinearity = 1
                    f.iip3_dbm = float(fe.iip3_dbm)
                if fe.adc_bits is not None:
                    f.has_adc = 1
                    f.adc_bits = int(fe.adc_bits)
                    f.adc_full_scale_v = float(fe.adc_full_scale_v)
        self._keep.append(bands)
        c.n_bands = len(r.bands)
        c.bands = C.cast(bands, C.POINTER(A.BandCfg))


def to_c(scene: Scene, time_base: int = A.LPK_TIME_BASE_SCENE,
         default_signal_epoch_unix: float = 0.0) -> CScene:
    return CScene(scene, time_base, default_signal_epoch_unix)


def replace(obj, **kw):
    return dataclasses.replace(obj, **kw)
