"""ctypes mirror of include/lipika_scene.h.

The structs restate the reference's TOML schema (src/config/mod.rs:52-460)
as flat C data. They are shared by the product host (liblipika_cuda.so) and,
in tests only, by the CPU oracle.
"""
import ctypes as C

LPK_TRAJ_STATIONARY_GEODETIC = 0
LPK_TRAJ_STATIONARY_ECEF = 1
LPK_TRAJ_CIRCULAR_KEPLERIAN = 2
LPK_TRAJ_TLE = 3
LPK_TRAJ_RINEX_NAV = 4

LPK_SIG_CW = 0
LPK_SIG_BPSK = 1
LPK_SIG_OOK = 2
LPK_SIG_QAM16 = 3
LPK_SIG_CA_CODE = 4

LPK_NAV_OFF = 0
LPK_NAV_DUMMY = 1
LPK_NAV_FULL = 2

LPK_TIME_BASE_SCENE = 0
LPK_TIME_BASE_ABSOLUTE = 1

LPK_SCENE_DEVICE_TABLES = 1  # lpk_scene_cfg.flags


class TrajectoryCfg(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("reserved", C.c_int32),
        ("lat_deg", C.c_double), ("lon_deg", C.c_double), ("h_m", C.c_double),
        ("x_m", C.c_double), ("y_m", C.c_double), ("z_m", C.c_double),
        ("semi_major_axis_m", C.c_double), ("inclination_deg", C.c_double),
        ("raan_deg", C.c_double), ("true_anomaly_deg_at_epoch", C.c_double),
        ("epoch_unix", C.c_double),
    ]


class TransmitterCfg(C.Structure):
    _fields_ = [
        ("carrier_hz", C.c_double), ("tx_power_dbw", C.c_double),
        ("kind", C.c_int32), ("has_bandwidth", C.c_int32), ("bandwidth_hz", C.c_double),
        ("trajectory", TrajectoryCfg),
        ("has_signal_epoch", C.c_int32), ("has_gate", C.c_int32),
        ("signal_epoch_unix", C.c_double),
        ("gate_period_s", C.c_double), ("gate_epoch_unix", C.c_double),
        ("gate_n_bursts", C.c_int32), ("reserved0", C.c_int32),
        ("gate_bursts", C.POINTER(C.c_double)),
        ("baseband_offset_hz", C.c_double),
        ("rate_hz", C.c_double),
        ("payload_n", C.c_int64), ("payload_seed", C.c_uint64),
        ("sync_n", C.c_int32), ("reserved1", C.c_int32),
        ("sync_word", C.POINTER(C.c_int8)),
        ("prn", C.c_int32), ("nav", C.c_int32),
        ("ca_epoch_unix", C.c_double), ("nav_seed", C.c_uint64),
    ]


class ClockCfg(C.Structure):
    _fields_ = [
        ("allan_deviation_1s", C.c_double), ("flicker_floor", C.c_double),
        ("frequency_offset_y0", C.c_double), ("initial_time_offset_s", C.c_double),
    ]


class FrontendCfg(C.Structure):
    _fields_ = [
        ("has_antenna", C.c_int32), ("has_cutoff", C.c_int32),
        ("peak_dbi", C.c_double), ("horizon_dbi", C.c_double), ("fb_db", C.c_double),
        ("cutoff_deg", C.c_double),
        ("has_gain", C.c_int32), ("has_nonlinearity", C.c_int32),
        ("gain_db", C.c_double), ("iip3_dbm", C.c_double),
        ("has_adc", C.c_int32), ("adc_bits", C.c_uint32), ("adc_full_scale_v", C.c_double),
    ]


class BandCfg(C.Structure):
    _fields_ = [
        ("lo_carrier_hz", C.c_double), ("sample_rate_hz", C.c_double),
        ("noise_temperature_k", C.c_double),
        ("has_noise_power", C.c_int32), ("has_bandwidth", C.c_int32),
        ("noise_power_w", C.c_double), ("bandwidth_hz", C.c_double),
        ("has_frontend", C.c_int32), ("reserved", C.c_int32),
        ("frontend", FrontendCfg),
    ]


class ReceiverCfg(C.Structure):
    _fields_ = [
        ("trajectory", TrajectoryCfg), ("clock", ClockCfg),
        ("n_bands", C.c_int32), ("reserved", C.c_int32),
        ("bands", C.POINTER(BandCfg)),
    ]


class SceneCfg(C.Structure):
    _fields_ = [
        ("epoch_unix", C.c_double), ("duration_s", C.c_double),
        ("gps_utc_offset_s", C.c_double), ("default_signal_epoch_unix", C.c_double),
        ("time_base", C.c_int32), ("n_transmitters", C.c_int32),
        ("transmitters", C.POINTER(TransmitterCfg)),
        ("n_receivers", C.c_int32), ("flags", C.c_int32),
        ("receivers", C.POINTER(ReceiverCfg)),
    ]
