"""Scene fixtures used by the parity tests.

The small scenes restate the inline TOML fixtures of the reference's
integration tests (tests/multi_transmitter_summation.rs:14-132,
tests/streaming_chunk_invariance.rs:260-303, tests/ook_qam16_end_to_end.rs:
403-439) with the same parameter values; the `config_*` builders are the
BASELINE workloads, defined in lipika_b200.workloads and re-exported here.
"""
from __future__ import annotations

from lipika_b200 import config as cfg

NO_TX = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.5

[[receiver]]
name = "lab"
trajectory = { kind = "stationary_geodetic", lat_deg = 55.86, lon_deg = -4.25, h_m = 10.0 }
clock = { allan_deviation_1s = 0.0 }
[[receiver.band]]
band_id = "test"
lo_carrier_hz = 1_000_000_000.0
sample_rate_hz = 1_000_000.0
noise_power_w = 1.0e-15
"""

TWO_TX = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.5

[[transmitter]]
name = "alpha"
carrier_hz = 1_000_000_000.0
tx_power_dbw = 30.0
kind = "cw"
baseband_offset_hz = 0.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 1000.0 }

[[transmitter]]
name = "beta"
carrier_hz = 1_005_000_000.0
tx_power_dbw = 30.0
kind = "cw"
baseband_offset_hz = 0.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 1000.0, z_m = 1000.0 }

[[receiver]]
name = "lab"
trajectory = { kind = "stationary_geodetic", lat_deg = 55.86, lon_deg = -4.25, h_m = 10.0 }
clock = { allan_deviation_1s = 0.0 }
[[receiver.band]]
band_id = "test"
lo_carrier_hz = 1_000_000_000.0
sample_rate_hz = 1_000_000.0
noise_power_w = 1.0e-15
"""

BPSK = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.05

[[transmitter]]
name = "beacon"
carrier_hz = 1_000_000_000.0
tx_power_dbw = 30.0
kind = "bpsk"
bit_rate_bps = 100_000.0
payload_bits = 6000
payload_seed = 7
sync_word = [1, -1, 1, 1, -1, -1, 1, -1]
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 0.0 }

[[receiver]]
name = "lab"
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 100000.0 }
clock = { allan_deviation_1s = 0.0 }
[[receiver.band]]
band_id = "test"
lo_carrier_hz = 1_000_000_000.0
sample_rate_hz = 1_000_000.0
noise_power_w = 1.0e-18
"""

CW_TWO_CLOCKS = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.02

[[transmitter]]
name = "cw"
carrier_hz = 1000000.0
tx_power_dbw = 0.0
kind = "cw"
baseband_offset_hz = 0.0
trajectory = { kind = "stationary_ecef", x_m = 6478137.0, y_m = 0.0, z_m = 0.0 }

[[receiver]]
name = "rxa"
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 0.0 }
clock = { initial_time_offset_s = 0.0 }
[[receiver.band]]
band_id = "b"
lo_carrier_hz = 1000000.0
sample_rate_hz = 100000.0
noise_power_w = 1.0e-30

[[receiver]]
name = "rxb"
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 0.0 }
clock = { initial_time_offset_s = 1.3e-7 }
[[receiver.band]]
band_id = "b"
lo_carrier_hz = 1000000.0
sample_rate_hz = 100000.0
noise_power_w = 1.0e-30
"""

STREAMING = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.05

[[transmitter]]
name = "a0"
carrier_hz = 1_000_000_000.0
tx_power_dbw = 30.0
kind = "cw"
baseband_offset_hz = 1234.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 1000.0 }

[[transmitter]]
name = "a1"
carrier_hz = 1_000_050_000.0
tx_power_dbw = 28.0
kind = "cw"
baseband_offset_hz = -777.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 2000.0, z_m = 500.0 }

[[transmitter]]
name = "b0"
carrier_hz = 1_500_000_000.0
tx_power_dbw = 30.0
kind = "cw"
baseband_offset_hz = 333.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 1000.0, z_m = 1000.0 }

[[receiver]]
name = "rx"
trajectory = { kind = "stationary_geodetic", lat_deg = 55.86, lon_deg = -4.25, h_m = 10.0 }
clock = { allan_deviation_1s = 1e-9, frequency_offset_y0 = 0.5e-6, initial_time_offset_s = 1e-7 }
[[receiver.band]]
band_id = "a"
lo_carrier_hz = 1_000_000_000.0
sample_rate_hz = 1_000_000.0
noise_power_w = 1.0e-15
[[receiver.band]]
band_id = "b"
lo_carrier_hz = 1_500_000_000.0
sample_rate_hz = 200_000.0
noise_power_w = 1.0e-15
"""

OOK_QAM_TEMPLATE = """
[scene]
epoch_unix = 1717260840.0
duration_s = 0.05

[[transmitter]]
name = "src"
carrier_hz = 1_000_000_000.0
tx_power_dbw = 30.0
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 0.0 }
@SIGNAL@

[[receiver]]
name = "lab"
trajectory = { kind = "stationary_ecef", x_m = 6378137.0, y_m = 0.0, z_m = 100000.0 }
clock = { allan_deviation_1s = 0.0 }
[[receiver.band]]
band_id = "test"
lo_carrier_hz = 1_000_000_000.0
sample_rate_hz = 1_000_000.0
noise_power_w = 1.0e-30
"""
SIG_CW = 'kind = "cw"\nbaseband_offset_hz = 0.0'
SIG_OOK = ('kind = "ook"\nbit_rate_bps = 100_000.0\npayload_bits = 6000\npayload_seed = 7\n'
           'sync_word = [1, 0, 1, 1, 0, 0, 1, 0]')
SIG_QAM16 = ('kind = "qam16"\nsymbol_rate_baud = 100_000.0\npayload_symbols = 6000\npayload_seed = 7\n'
             'sync_word = [0, 0, 0, 0, 1, 0, 1, 0]')


def parse(text: str) -> cfg.Scene:
    return cfg.scene_from_toml_str(text)


# The BASELINE workloads live in the package (bench.py and smoke() use them);
# re-exported here for the tests.
from lipika_b200.workloads import (EPOCH, GLASGOW_CLOCK, C1_LEO, C1_SYNC, config_c0, config_c1,  # noqa: E402,F401
                                   config_c2, config_c3, config_c4)
