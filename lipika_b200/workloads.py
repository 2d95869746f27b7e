"""The BASELINE workloads as scene descriptions (lipika_b200.config.Scene).

Each builder restates one of the five synthetic scenes the benchmark and the
parity tests run, with the parameters the workload text leaves open fixed
here and recorded (LEO RAAN 100 deg and true anomaly 270 deg for the
dual-band beacon; seeded receivers, clocks, orbits and payloads for the
24- and 64-transmitter scenes). Scene epoch 1717260840.0 (2024-06-01T16:54Z).

  config_c0  one CW GPS-altitude transmitter, one Glasgow receiver, 1 s at 2.048 MS/s
  config_c1  dual-band 120 s: 437 MHz BPSK LEO beacon (48 kS/s band) + C/A PRN 1-6 (2.048 MS/s band)
  config_c2  24 C/A x 32 seeded receivers with 1-3 bands of uneven rate, 30 s
  config_c3  config_c1 extended to 600 s with the L1 band at 8.184 MS/s (long coherent scene)
  config_c4  64 transmitters (CW / OOK / 16-QAM / C/A) x 16 receivers, 60 s at 2.048 MS/s
"""
from __future__ import annotations

import numpy as np

from . import config as cfg

EPOCH = 1717260840.0

def _kepler(a, inc, raan, ta, epoch=EPOCH):
    return cfg.Trajectory("circular_keplerian", {
        "semi_major_axis_m": a, "inclination_deg": inc, "raan_deg": raan,
        "true_anomaly_deg_at_epoch": ta, "epoch_unix": epoch})


def _glasgow():
    return cfg.Trajectory("stationary_geodetic", {"lat_deg": 55.86, "lon_deg": -4.25, "h_m": 10.0})


GLASGOW_CLOCK = cfg.Clock(allan_deviation_1s=1e-11, frequency_offset_y0=0.5e-6)


def config_c0(duration_s: float = 1.0, clock: cfg.Clock | None = None, noise: bool = True) -> cfg.Scene:
    """One CW GPS-altitude transmitter, one Glasgow receiver, 2.048 MS/s."""
    tx = cfg.Transmitter(name="cw_l1", carrier_hz=1575.42e6, kind="cw",
                         params={"baseband_offset_hz": 0.0},
                         trajectory=_kepler(26_578_137.0, 55.0, 0.0, 30.0), tx_power_dbw=27.0)
    band = cfg.Band("l1", 1575.42e6, 2.048e6, 290.0, None if noise else 0.0)
    rx = cfg.Receiver("glasgow", _glasgow(), clock or GLASGOW_CLOCK, [band])
    return cfg.Scene(EPOCH, duration_s, [tx], [rx])


C1_SYNC = [-1, 1, 1, -1, 1, -1, -1, 1]
C1_LEO = dict(a=6_791_000.0, inc=51.6, raan=100.0, ta=270.0)  # RAAN/TA fixed here


def config_c1(duration_s: float = 120.0, clock: cfg.Clock | None = None, noise: bool = True,
              l1_rate: float = 2.048e6) -> cfg.Scene:
    """Dual-band plain scene: a 437 MHz BPSK LEO beacon + C/A PRN 1-6."""
    txs = [cfg.Transmitter(
        name="uhf_beacon", carrier_hz=437e6, kind="bpsk",
        params={"bit_rate_bps": 9600.0, "payload_bits": 287_968, "payload_seed": 2026,
                "sync_word": C1_SYNC},
        trajectory=_kepler(C1_LEO["a"], C1_LEO["inc"], C1_LEO["raan"], C1_LEO["ta"]), tx_power_dbw=0.0)]
    for k in range(6):
        txs.append(cfg.Transmitter(
            name=f"gps_prn{k + 1:02d}", carrier_hz=1575.42e6, kind="ca_code",
            params={"prn": k + 1, "epoch_unix": EPOCH, "nav": "dummy", "nav_seed": 0},
            trajectory=_kepler(26_578_137.0, 55.0, 60.0 * k, 30.0 + 50.0 * k), tx_power_dbw=27.0))
    bands = [cfg.Band("uhf_obs", 437e6, 48_000.0, 290.0, None if noise else 0.0),
             cfg.Band("gnss_l1", 1575.42e6, l1_rate, 290.0, None if noise else 0.0)]
    rx = cfg.Receiver("glasgow", _glasgow(), clock or GLASGOW_CLOCK, bands)
    return cfg.Scene(EPOCH, duration_s, txs, [rx])


def config_c3(duration_s: float = 600.0, clock: cfg.Clock | None = None, noise: bool = True) -> cfg.Scene:
    """Long coherent scene: the dual-band scene over 600 s with the L1 band
    at 8.184 MS/s (4.91e9 L1 samples x 6 C/A transmitters + 2.88e7 UHF
    samples x 1 BPSK beacon = 2.95e10 tx-rx samples)."""
    return config_c1(duration_s=duration_s, clock=clock, noise=noise, l1_rate=8.184e6)


def config_c2(duration_s: float = 30.0, seed: int = 2026, n_rx: int = 32, noise: bool = True,
              clock_walk: bool = True) -> cfg.Scene:
    """Batched uneven scene: 24 C/A (6 planes x 4 slots), seeded receivers."""
    rng = np.random.default_rng(seed)
    txs = []
    prn = 1
    for p in range(6):
        for s in range(4):
            txs.append(cfg.Transmitter(
                name=f"gps_p{p}s{s}", carrier_hz=1575.42e6, kind="ca_code",
                params={"prn": prn, "epoch_unix": EPOCH, "nav": "dummy", "nav_seed": 0},
                trajectory=_kepler(26_578_137.0, 55.0, 60.0 * p, 90.0 * s + 15.0 * p), tx_power_dbw=27.0))
            prn += 1
    rates = [48_000.0, 250_000.0, 2.048e6, 4.096e6]
    rxs = []
    for r in range(n_rx):
        lat = float(rng.uniform(-70, 70))
        lon = float(rng.uniform(-180, 180))
        h = float(rng.uniform(0, 500))
        allan = float(10 ** rng.uniform(-12, -10)) if clock_walk else 0.0
        y0 = float(rng.uniform(-1e-6, 1e-6))
        nb = int(rng.integers(1, 4))
        bands = [cfg.Band(f"b{b}", 1575.42e6, float(rates[int(rng.integers(0, 4))]), 290.0,
                          None if noise else 0.0) for b in range(nb)]
        rxs.append(cfg.Receiver(f"rx{r:02d}", cfg.Trajectory("stationary_geodetic",
                                {"lat_deg": lat, "lon_deg": lon, "h_m": h}),
                                cfg.Clock(allan_deviation_1s=allan, frequency_offset_y0=y0), bands))
    return cfg.Scene(EPOCH, duration_s, txs, rxs)


def config_c4(duration_s: float = 60.0, seed: int = 2026, n_rx: int = 16, noise: bool = True,
              lo_hz: float = 1575.42e6, n_tx: int = 64) -> cfg.Scene:
    """n_tx transmitters (64 by default: 16 each CW / OOK 1 kbit/s / 16-QAM
    10 ksym/s / C/A PRN 1-16; a quarter of n_tx of each kind, PRNs cycling
    1-32)."""
    assert n_tx % 4 == 0
    rng = np.random.default_rng(seed)
    txs = []
    for k in range(n_tx):
        kind = ("cw", "ook", "qam16", "ca_code")[k // (n_tx // 4)]
        a = float(rng.uniform(6_900_000.0, 26_600_000.0))
        inc = float(rng.uniform(0.0, 98.0))
        raan = float(rng.uniform(0.0, 360.0))
        ta = float(rng.uniform(0.0, 360.0))
        off = float(rng.uniform(-0.8e6, 0.8e6))
        if kind == "cw":
            params = {"baseband_offset_hz": float(rng.uniform(-2e3, 2e3))}
            carrier = lo_hz + off
        elif kind == "ook":
            params = {"bit_rate_bps": 1000.0, "payload_bits": int(duration_s * 1000) + 64,
                      "payload_seed": int(rng.integers(0, 2**31)), "sync_word": [1, 0, 1, 1, 0, 0, 1, 0]}
            carrier = lo_hz + off
        elif kind == "qam16":
            params = {"symbol_rate_baud": 10_000.0, "payload_symbols": int(duration_s * 10_000) + 64,
                      "payload_seed": int(rng.integers(0, 2**31)), "sync_word": [0, 0, 0, 0, 1, 0, 1, 0]}
            carrier = lo_hz + off
        else:
            params = {"prn": 1 + (k - 3 * n_tx // 4) % 32, "epoch_unix": EPOCH, "nav": "dummy", "nav_seed": 0}
            carrier = lo_hz
        txs.append(cfg.Transmitter(name=f"tx{k:02d}_{kind}" if n_tx <= 100 else f"tx{k:03d}_{kind}", carrier_hz=carrier, kind=kind, params=params,
                                   trajectory=_kepler(a, inc, raan, ta), tx_power_dbw=20.0))
    rxs = []
    for r in range(n_rx):
        traj = cfg.Trajectory("stationary_geodetic", {"lat_deg": float(rng.uniform(-70, 70)),
                                                      "lon_deg": float(rng.uniform(-180, 180)),
                                                      "h_m": float(rng.uniform(0, 500))})
        rxs.append(cfg.Receiver(f"rx{r:02d}", traj, cfg.Clock(allan_deviation_1s=1e-11,
                                                             frequency_offset_y0=float(rng.uniform(-1e-6, 1e-6))),
                                [cfg.Band("l1", lo_hz, 2.048e6, 290.0, None if noise else 0.0)]))
    return cfg.Scene(EPOCH, duration_s, txs, rxs)
