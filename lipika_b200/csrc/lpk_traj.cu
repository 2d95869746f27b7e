// lpk_traj.cu — trajectory tables of circular Keplerian orbits built on the
// GPU: PrecomputedTrajectory::sample (src/geometry/precomputed.rs:47-70)
// over CircularKeplerian::position_ecef (src/geometry/kepler.rs:32-85),
// one thread per (orbit, grid point).
//
// The host's kepler() (lpk_host.cpp) evaluates the same expression. The
// per-orbit constants (mean motion, radians of the angles, their sines and
// cosines) are computed once on the host with its libm and passed in, and
// every per-point operation is spelled with explicit rounding in the host's
// order, so a device-built table differs from a host-built one only where
// the GPU's sin/cos of the two per-point angles differ from the host's in
// the last ulp (~1e-9 m of position).
#include <cmath>
#include <vector>

#include "lpk_internal.h"

namespace lpk {

namespace {

constexpr double kKeplerGm = 3.986005e14;  // src/geometry/kepler.rs:12

__global__ void __launch_bounds__(256)
k_kepler_table(const DevOrbit *__restrict__ orbits, int32_t n_orbits, double t0, double dt, int64_t n,
               double *__restrict__ out) {
    const int64_t total = (int64_t)n_orbits * n;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total;
         id += (int64_t)gridDim.x * blockDim.x) {
        const int o = (int)(id / n);
        const int64_t i = id - (int64_t)o * n;
        const DevOrbit k = orbits[o];
        const double t = __dadd_rn(t0, __dmul_rn((double)i, dt));  // start + i·dt (precomputed.rs)
        double x, y, z;
        kepler_at(k, __dsub_rn(t, k.epoch), x, y, z);
        double *dst = out + (int64_t)o * 3 * n;
        dst[i] = x;
        dst[n + i] = y;
        dst[2 * n + i] = z;
    }
}

inline double deg2rad(double deg) { return deg * (M_PI / 180.0); }  // f64::to_radians

}  // namespace

// The per-orbit part of kepler.rs:32-85 with the host's libm (the order of
// the host's kepler() in lpk_host.cpp); false for a non-positive or
// non-finite radius or a non-finite angle or epoch.
bool make_orbit(const lpk_kepler_orbit &k, DevOrbit &o) {
    const double r = k.semi_major_axis_m;
    if (!(r > 0.0) || !std::isfinite(r) || !std::isfinite(k.inclination_deg) || !std::isfinite(k.raan_deg) ||
        !std::isfinite(k.true_anomaly_deg_at_epoch) || !std::isfinite(k.epoch_unix))
        return false;
    const double inc = deg2rad(k.inclination_deg), om = deg2rad(k.raan_deg);
    o = DevOrbit{r, std::sqrt(kKeplerGm / (r * r * r)), deg2rad(k.true_anomaly_deg_at_epoch), std::sin(inc),
                 std::cos(inc), std::sin(om), std::cos(om), k.epoch_unix};
    return true;
}

}  // namespace lpk

using namespace lpk;

extern "C" lpk_status lpk_kepler_tables(lpk_ctx *c, const lpk_kepler_orbit *orbits, int32_t n_orbits, double t0_unix,
                                        double dt_s, int64_t n_points, double *grid_xyz) {
    if (!c) return fail(nullptr, LPK_EINVAL, "ctx is NULL");
    if (n_orbits < 0 || n_points < 0) return fail(c, LPK_EINVAL, "negative orbit or point count");
    if (n_orbits == 0 || n_points == 0) return LPK_OK;
    if (!orbits || !grid_xyz) return fail(c, LPK_EINVAL, "orbits or grid_xyz is NULL");
    if (!std::isfinite(t0_unix) || !(dt_s > 0.0) || !std::isfinite(dt_s))
        return fail(c, LPK_EINVAL, "t0 must be finite and dt positive");
    if (n_points > ((int64_t)1 << 31)) return fail(c, LPK_EINVAL, "too many grid points");
    std::vector<DevOrbit> h((size_t)n_orbits);
    for (int32_t o = 0; o < n_orbits; ++o)
        if (!make_orbit(orbits[o], h[o])) return fail(c, LPK_EINVAL, "bad orbit (radius must be positive)");
    cudaSetDevice(c->device);
    const size_t obytes = sizeof(DevOrbit) * (size_t)n_orbits;
    const size_t gbytes = sizeof(double) * 3 * (size_t)n_points * (size_t)n_orbits;
    void *d_orb = nullptr, *d_grid = nullptr;
    cudaError_t e = pool_alloc(c, &d_orb, obytes);
    if (e == cudaSuccess) e = pool_alloc(c, &d_grid, gbytes);
    if (e != cudaSuccess) {
        if (d_orb) pool_free(c, d_orb);
        return fail(c, LPK_ENOMEM, "trajectory table allocation failed");
    }
    e = cudaMemcpyAsync(d_orb, h.data(), obytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        const int64_t total = (int64_t)n_orbits * n_points;
        const int64_t want = (total + 255) / 256;
        const unsigned grid = (unsigned)(want < (int64_t)sms * 16 ? want : (int64_t)sms * 16);
        k_kepler_table<<<grid, 256, 0, c->stream>>>((const DevOrbit *)d_orb, n_orbits, t0_unix, dt_s, n_points,
                                                    (double *)d_grid);
        e = cudaGetLastError();
        if (e == cudaSuccess) c->launches += 1;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(grid_xyz, d_grid, gbytes, cudaMemcpyDeviceToHost, c->stream);
    pool_free(c, d_grid);
    pool_free(c, d_orb);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "trajectory tables");
    return LPK_OK;
}
