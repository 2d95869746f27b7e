"""Trajectory tables built on the GPU (lpk_kepler_tables): the positions of
PrecomputedTrajectory::sample over CircularKeplerian::position_ecef
(src/geometry/precomputed.rs:47-70, src/geometry/kepler.rs:32-85), checked
against the host-built tables, which are bit-identical to the oracle's
(test_abi_cpu.py), and through the fan-out."""
import time

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from tests import scenes
from tests.test_abi_cpu import HostScene

pytestmark = pytest.mark.gpu

POS_TOL_M = 1e-6  # ~1e-9 m expected: last-ulp differences of sin/cos only


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


def _orbits(scene):
    out, idx = [], []
    for i, t in enumerate(scene.transmitters):
        tr = t.trajectory
        if tr.kind == "circular_keplerian":
            k = tr.params
            out.append(N.KeplerOrbit(k["semi_major_axis_m"], k["inclination_deg"], k["raan_deg"],
                                     k["true_anomaly_deg_at_epoch"], k["epoch_unix"]))
            idx.append(i)
    return (N.KeplerOrbit * len(out))(*out), idx


def test_device_tables_match_host_tables(ctx):
    sc = scenes.config_c4(duration_s=30.0, n_rx=1)  # 64 orbits from 6,900 to 26,600 km
    hs = HostScene(sc)
    orbits, idx = _orbits(sc)
    d0 = hs.tx(idx[0])
    n = d0.grid_n
    grid = np.zeros(len(idx) * 3 * n)
    ctx.check(N.lib().lpk_kepler_tables(ctx.h, orbits, len(idx), d0.grid_t0_unix, d0.grid_dt_s, n,
                                        grid.ctypes.data_as(N._D)))
    worst, same = 0.0, 0
    for j, i in enumerate(idx):
        d = hs.tx(i)
        assert d.grid_n == n and d.grid_t0_unix == d0.grid_t0_unix
        host = np.ctypeslib.as_array(d.grid_xyz, shape=(3 * n,))
        dev = grid[j * 3 * n:(j + 1) * 3 * n]
        worst = max(worst, float(np.max(np.abs(dev - host))))
        same += int(np.sum(dev == host))
    print(f"device vs host tables: {len(idx)} orbits x {n} points, max |diff| {worst:.3e} m, "
          f"{same / (len(idx) * 3 * n):.4f} of entries bit-identical")
    assert worst <= POS_TOL_M
    assert same > 0.5 * len(idx) * 3 * n


def test_device_tables_through_the_fan_out(ctx):
    sc = scenes.config_c1(duration_s=2.0, noise=False)
    ctx2 = N.Context(0)  # a context holds one uploaded scene
    host = P.Prepared(sc, ctx)
    dev = P.Prepared(sc, ctx2, device_tables=True)
    for w, (r, b) in enumerate(host.work()):
        outs = []
        for prep in (host, dev):
            chunks = []
            res = prep.generate_band(r, b, 7, w, 1 << 18, lambda c: chunks.append(c.copy()) and False, noise=False)
            outs.append((np.concatenate(chunks), [bool(res.unoccluded[k]) for k in range(res.n_active)]))
        (a, fa), (b_, fb) = outs
        scale = max(float(np.max(np.abs(a))), 1e-30)
        assert fa == fb
        assert float(np.max(np.abs(a.astype(np.complex128) - b_))) <= 1e-5 * scale
    host.close()
    dev.close()
    ctx2.close()


def test_device_tables_time_for_a_large_sky(ctx):
    sky = 1000
    rng = np.random.default_rng(2026)
    orbits = (N.KeplerOrbit * sky)(*[N.KeplerOrbit(float(rng.uniform(6.9e6, 2.66e7)), float(rng.uniform(0, 98)),
                                                   float(rng.uniform(0, 360)), float(rng.uniform(0, 360)),
                                                   1717260840.0) for _ in range(sky)])
    n = 12_102  # 120 s at 10 ms with the 0.5 s pads
    grid = np.zeros(sky * 3 * n)
    L = N.lib()
    ctx.check(L.lpk_kepler_tables(ctx.h, orbits, sky, 1717260839.5, 0.01, n, grid.ctypes.data_as(N._D)))
    t = time.perf_counter()
    ctx.check(L.lpk_kepler_tables(ctx.h, orbits, sky, 1717260839.5, 0.01, n, grid.ctypes.data_as(N._D)))
    dt = time.perf_counter() - t
    g = grid.reshape(sky, 3, n)
    r = np.sqrt(g[:, 0] ** 2 + g[:, 1] ** 2 + g[:, 2] ** 2)
    a = np.array([o.semi_major_axis_m for o in orbits])
    assert np.max(np.abs(r / a[:, None] - 1.0)) < 1e-12  # circular: |P| = a everywhere
    print(f"{sky} orbits x {n} points on the GPU (to host memory): {dt * 1e3:.1f} ms")


def test_kepler_tables_reject_bad_arguments(ctx):
    L = N.lib()
    o = (N.KeplerOrbit * 1)(N.KeplerOrbit(7e6, 50.0, 0.0, 0.0, 0.0))
    g = np.zeros(6)
    assert L.lpk_kepler_tables(ctx.h, o, 1, 0.0, 0.0, 2, g.ctypes.data_as(N._D)) == N.LPK_EINVAL
    assert L.lpk_kepler_tables(ctx.h, o, 1, 0.0, 0.01, 2, None) == N.LPK_EINVAL
    bad = (N.KeplerOrbit * 1)(N.KeplerOrbit(-1.0, 50.0, 0.0, 0.0, 0.0))
    assert L.lpk_kepler_tables(ctx.h, bad, 1, 0.0, 0.01, 2, g.ctypes.data_as(N._D)) == N.LPK_EINVAL
    assert L.lpk_kepler_tables(ctx.h, o, 0, 0.0, 0.01, 2, g.ctypes.data_as(N._D)) == N.LPK_OK
