/*
 * lipika_scene.h — plain-C description of a lipika scene.
 *
 * These structs restate the TOML schema of the reference
 * (src/config/mod.rs:52-460) as flat C data so that a host written in any
 * language can describe a scene across a C ABI. They carry no behaviour:
 * the product host (liblipika_cuda.so, lpk_host_*) and the CPU oracle
 * (oracle/, test infrastructure only) each build their own tables from them.
 *
 * Every "has_*" flag mirrors an `Option<_>` of the reference schema; the
 * default values a missing TOML key takes are applied by whoever fills the
 * struct (lipika_b200/config.py does it for Python callers).
 */
#ifndef LIPIKA_SCENE_H
#define LIPIKA_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* TrajectoryConfig variants (src/config/mod.rs:429-445). TLE (SGP4) and
 * RINEX broadcast ephemerides are not built by this backend. */
enum {
    LPK_TRAJ_STATIONARY_GEODETIC = 0,
    LPK_TRAJ_STATIONARY_ECEF = 1,
    LPK_TRAJ_CIRCULAR_KEPLERIAN = 2,
    LPK_TRAJ_TLE = 3,
    LPK_TRAJ_RINEX_NAV = 4
};

typedef struct lpk_trajectory_cfg {
    int32_t kind;
    int32_t reserved;
    /* stationary_geodetic */
    double lat_deg, lon_deg, h_m;
    /* stationary_ecef */
    double x_m, y_m, z_m;
    /* circular_keplerian */
    double semi_major_axis_m, inclination_deg, raan_deg, true_anomaly_deg_at_epoch, epoch_unix;
} lpk_trajectory_cfg;

/* SignalKind variants (src/config/mod.rs:196-222). */
enum { LPK_SIG_CW = 0, LPK_SIG_BPSK = 1, LPK_SIG_OOK = 2, LPK_SIG_QAM16 = 3, LPK_SIG_CA_CODE = 4 };
/* NavMode (src/config/mod.rs:224-237). */
enum { LPK_NAV_OFF = 0, LPK_NAV_DUMMY = 1, LPK_NAV_FULL = 2 };

typedef struct lpk_transmitter_cfg {
    double carrier_hz;
    double tx_power_dbw;
    int32_t kind;               /* LPK_SIG_* */
    int32_t has_bandwidth;
    double bandwidth_hz;
    lpk_trajectory_cfg trajectory;
    int32_t has_signal_epoch;
    int32_t has_gate;
    double signal_epoch_unix;
    /* gate (src/config/mod.rs:121-143) */
    double gate_period_s;
    double gate_epoch_unix;
    int32_t gate_n_bursts;
    int32_t reserved0;
    const double *gate_bursts;  /* gate_n_bursts pairs (offset_s, duration_s) */
    /* cw */
    double baseband_offset_hz;
    /* bpsk / ook: bit_rate_bps; qam16: symbol_rate_baud */
    double rate_hz;
    int64_t payload_n;          /* payload_bits / payload_symbols */
    uint64_t payload_seed;
    int32_t sync_n;
    int32_t reserved1;
    const int8_t *sync_word;    /* bpsk: ±1; ook, qam16: 0/1 */
    /* ca_code */
    int32_t prn;
    int32_t nav;                /* LPK_NAV_* */
    double ca_epoch_unix;
    uint64_t nav_seed;
} lpk_transmitter_cfg;

/* NodeClockSpec (src/clock/mod.rs:19-35). */
typedef struct lpk_clock_cfg {
    double allan_deviation_1s;
    double flicker_floor;
    double frequency_offset_y0;
    double initial_time_offset_s;
} lpk_clock_cfg;

/* FrontendConfig (src/config/mod.rs:311-360). */
typedef struct lpk_frontend_cfg {
    int32_t has_antenna;
    int32_t has_cutoff;
    double peak_dbi, horizon_dbi, fb_db, cutoff_deg;
    int32_t has_gain;
    int32_t has_nonlinearity;
    double gain_db;
    double iip3_dbm;
    int32_t has_adc;
    uint32_t adc_bits;
    double adc_full_scale_v;
} lpk_frontend_cfg;

/* ReceiverBandConfig (src/config/mod.rs:282-307). */
typedef struct lpk_band_cfg {
    double lo_carrier_hz;
    double sample_rate_hz;
    double noise_temperature_k;
    int32_t has_noise_power;
    int32_t has_bandwidth;
    double noise_power_w;
    double bandwidth_hz;
    int32_t has_frontend;
    int32_t reserved;
    lpk_frontend_cfg frontend;
} lpk_band_cfg;

/* ReceiverConfig (src/config/mod.rs:271-280). */
typedef struct lpk_receiver_cfg {
    lpk_trajectory_cfg trajectory;
    lpk_clock_cfg clock;
    int32_t n_bands;
    int32_t reserved;
    const lpk_band_cfg *bands;
} lpk_receiver_cfg;

/* How emissions are tied to time (src/pipeline.rs:124-139). */
enum { LPK_TIME_BASE_SCENE = 0, LPK_TIME_BASE_ABSOLUTE = 1 };

/* SceneConfig (src/config/mod.rs:52-69) plus the render's time base. */
typedef struct lpk_scene_cfg {
    double epoch_unix;
    double duration_s;
    double gps_utc_offset_s;
    double default_signal_epoch_unix;   /* used when time_base == ABSOLUTE */
    int32_t time_base;
    int32_t n_transmitters;
    const lpk_transmitter_cfg *transmitters;
    int32_t n_receivers;
    int32_t flags;                      /* LPK_SCENE_* below */
    const lpk_receiver_cfg *receivers;
} lpk_scene_cfg;

/* lpk_scene_cfg.flags: LPK_SCENE_DEVICE_TABLES builds the trajectory tables
 * of circular Keplerian transmitters on the GPU (lpk_kepler_tables) instead
 * of the host (needs a context). */
enum { LPK_SCENE_DEVICE_TABLES = 1 };

#ifdef __cplusplus
}
#endif
#endif /* LIPIKA_SCENE_H */
