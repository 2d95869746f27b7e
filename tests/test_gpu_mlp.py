"""The learned warm start of the converged emission solve: tensor-core
forward and training-gradient kernels against the CPU restatement, the
network's feature layer against its float64 restatement, the bounded
tensor-core wait's give-up path, the converged solver against the oracle's
80-bit solve, and what the scene's trained network gains over starting
where the reference starts (t - 70 ms) on the 64-transmitter x 16-receiver
scene."""
import ctypes as C

import numpy as np
import pytest

from lipika_b200 import native as N
from lipika_b200 import pipeline as P
from oracle import mlp_ref as M
from oracle import oracle as O
from tests import scenes

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-2     # norm-wise, per parameter tensor (BF16 operands, FP32 accumulation)
FORWARD_ATOL = 3e-3  # outputs are O(1)
# Converged FP64 solve vs the oracle's 80-bit solve: two ulps of the
# emission time, plus 2 fs for the oracle's own query epoch + t, which 80-bit
# arithmetic rounds to 1.2e-10 s (a few 1e-16 s of delay). Far below 1 ps.
TRUTH_ULP, TRUTH_ABS_S = 2, 2e-15


@pytest.fixture(scope="module")
def ctx():
    c = N.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def dual(ctx):
    sc = scenes.config_c1(duration_s=120.0)
    prep = P.Prepared(sc, ctx)
    d = prep.band_desc(0, 0, 2026, 0)
    yield sc, prep, np.array(d.rx_ecef[:]), d.epoch_unix
    prep.close()


@pytest.fixture(scope="module")
def sky():
    """The 64-transmitter x 16-receiver scene (60 s), its receivers, and a
    context of its own (a context holds one uploaded scene)."""
    c = N.Context(0)
    sc = scenes.config_c4(duration_s=60.0)
    prep = P.Prepared(sc, c)
    rx = np.array([prep.band_desc(r, 0, 2026, r).rx_ecef[:] for r in range(len(sc.receivers))])
    yield sc, prep, rx, c
    c.close()


def _params(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.3, 0.3, M.N_PARAMS).astype(np.float32)
    p[M.OFF_B1:M.OFF_W2] = rng.uniform(-0.1, 0.1, M.N_H)
    return p


def test_forward_matches_cpu_restatement(ctx):
    m = N.Mlp(ctx, seed=7)
    p = _params(1)
    m.set_params(p)
    rng = np.random.default_rng(2)
    x = rng.normal(size=(1000, M.N_F)).astype(np.float32)  # not a multiple of the 128-row tile
    y = m.forward(x)
    yr, _ = M.forward(p, x)
    assert np.max(np.abs(y - yr)) <= FORWARD_ATOL, np.max(np.abs(y - yr))
    m.close()


def test_forward_tile_edges_and_many_rows(ctx):
    """The tensor-core forward takes 128-row tiles: partial tiles, single
    rows and a 4M-row batch (checked on a sample of rows) all match the CPU
    restatement."""
    import time
    m = N.Mlp(ctx, seed=7)
    p = _params(3)
    m.set_params(p)
    rng = np.random.default_rng(4)
    for n in (1, 127, 128, 129, 4096 + 17):
        x = rng.normal(size=(n, M.N_F)).astype(np.float32)
        yr, _ = M.forward(p, x)
        assert np.max(np.abs(m.forward(x) - yr)) <= FORWARD_ATOL
    x = rng.normal(size=(1 << 22, M.N_F)).astype(np.float32)
    m.forward(x)
    t = time.perf_counter()
    y = m.forward(x)
    dt = time.perf_counter() - t
    pick = rng.choice(x.shape[0], 4096, replace=False)
    yr, _ = M.forward(p, x[pick])
    assert np.max(np.abs(y[pick] - yr)) <= FORWARD_ATOL
    print(f"forward of {x.shape[0]} rows with host copies: {dt * 1e3:.2f} ms")
    m.close()


@pytest.mark.parametrize("n", [128, 1000, 20000])
def test_gradient_matches_cpu_restatement(ctx, n):
    m = N.Mlp(ctx, seed=7)
    p = _params(3)
    m.set_params(p)
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, M.N_F)).astype(np.float32)
    t = rng.normal(size=n).astype(np.float32)
    loss, g = m.loss_grad(x, t)
    lr, gr = M.loss_grad(p, x, t)
    assert abs(loss - lr) <= 1e-4 * abs(lr)
    for name, a, b in M.TENSORS:
        err = np.linalg.norm(g[a:b] - gr[a:b]) / max(np.linalg.norm(gr[a:b]), 1e-30)
        assert err <= GRAD_RTOL, (name, n, err)
    m.close()


def test_wait_gives_up_and_context_stays_usable(ctx):
    """The inference kernel with its MMAs withheld: every bounded completion
    wait runs out (nothing is in flight), the call reports LPK_ETIMEDOUT,
    and the next real forward on the same context is correct."""
    import time
    m = N.Mlp(ctx, seed=7)
    p = _params(5)
    m.set_params(p)
    t0 = time.perf_counter()
    code = N.lib().lpk_mlp_wait_selftest(m.h, 5000, 1 << 12)
    assert code == N.LPK_ETIMEDOUT
    assert b"gave up" in N.lib().lpk_last_error(ctx.h)
    assert time.perf_counter() - t0 < 5.0
    x = np.random.default_rng(6).normal(size=(777, M.N_F)).astype(np.float32)
    yr, _ = M.forward(p, x)
    assert np.max(np.abs(m.forward(x) - yr)) <= FORWARD_ATOL
    m.close()


def test_features_match_cpu_restatement(sky):
    """The analytic feature layer (orbit state from the elements, line of
    sight, range, range rate) against its float64 restatement."""
    sc, prep, rx, ctx = sky
    txs, orbits = N.scene_orbits(sc)
    m = N.Mlp(ctx, seed=1)
    m.set_orbits(txs, orbits)
    t = np.linspace(0.0, 60.0, 4001)
    for k in (0, 17, 40, 63):
        o = orbits[k]
        f = m.features(txs[k], rx[k % len(rx)], sc.epoch_unix, t)
        fr, _ = M.features((o.semi_major_axis_m, o.inclination_deg, o.raan_deg, o.true_anomaly_deg_at_epoch),
                           o.epoch_unix, rx[k % len(rx)], sc.epoch_unix, t)
        scale = np.maximum(np.abs(fr), 1e-30)
        rel = np.abs(f - fr) / scale
        # FP32 features: relative error at float rounding, except where a
        # component crosses zero (then absolute, against the column's size)
        col = np.max(np.abs(fr), axis=0)
        assert np.all((rel <= 2e-6) | (np.abs(f - fr) <= 2e-6 * col)), k
    m.close()


@pytest.mark.parametrize("scheme", [N.LPK_ITER_FIXED_POINT, N.LPK_ITER_NEWTON])
def test_converged_solve_matches_oracle_truth(ctx, dual, scheme):
    sc, prep, rx, epoch = dual
    osc = O.Scene(sc)
    L = O.lib()
    t = np.linspace(0.0, 119.9, 997)
    obs = np.repeat(rx[:, None], len(t), axis=1).ravel().copy()
    for tx in range(len(sc.transmitters)):
        te, it, _ = N.solve_converged(ctx, tx, rx, epoch, t, tol=1e-16, max_iter=20, scheme=scheme)
        assert np.all(it > 0)
        ote, org = np.zeros(len(t)), np.zeros(len(t))
        oit = np.zeros(len(t), np.int32)
        L.orc_solve_converged(L.orc_scene_traj(osc.h, tx), O.dptr(obs), O.dptr(t), len(t), epoch, 1e-16, 30,
                              O.dptr(ote), O.dptr(org), oit.ctypes.data_as(C.POINTER(C.c_int32)))
        excess = np.abs(te - ote) - (TRUTH_ULP * np.spacing(np.abs(ote)) + TRUTH_ABS_S)
        assert np.max(excess) <= 0.0, (tx, np.max(np.abs(te - ote)))


def test_scene_solve_equals_pairwise_solve(ctx, dual):
    """lpk_solve_converged_scene (per-sample transmitter and receiver) gives
    the bits of lpk_solve_converged (one pair per call)."""
    sc, prep, rx, epoch = dual
    rng = np.random.default_rng(3)
    n = 5000
    tx = rng.integers(0, len(sc.transmitters), n).astype(np.int32)
    rx2 = np.stack([rx, rx + np.array([1000.0, -2000.0, 500.0])])
    ri = rng.integers(0, 2, n).astype(np.int32)
    t = rng.uniform(0.0, 119.0, n)
    te, it, _, ms = N.solve_converged_scene(ctx, tx, ri, rx2, epoch, t, tol=1e-14, scheme=N.LPK_ITER_NEWTON,
                                            start=N.LPK_START_GEOMETRIC)
    assert ms > 0.0
    for k in range(len(sc.transmitters)):
        for r in range(2):
            sel = (tx == k) & (ri == r)
            te1, it1, _ = N.solve_converged(ctx, k, rx2[r], epoch, t[sel], tol=1e-14, scheme=N.LPK_ITER_NEWTON,
                                            start=N.LPK_START_GEOMETRIC)
            assert np.array_equal(te[sel], te1) and np.array_equal(it[sel], it1)


def test_learned_start_cuts_iterations(sky):
    """One network for the 64 transmitters x 16 receivers, trained on 2^21
    converged solves, against the reference's start (t - 70 ms) and the
    table's geometric range, on fresh (transmitter, receiver, time) triples:
    fewer map evaluations than the lag start under both schemes, no more
    than the geometric start, every start converging to the same times."""
    sc, prep, rx, ctx = sky
    txs, orbits = N.scene_orbits(sc)
    m = N.Mlp(ctx, seed=5)
    curve = m.fit(txs, orbits, rx, sc.epoch_unix, 0.0, 60.0, n_train=1 << 21, steps=2000, batch=4096, lr=3e-3,
                  seed=9)
    assert curve[-50:].mean() < 0.01 * curve[:20].mean(), (curve[:5], curve[-5:])
    rng = np.random.default_rng(11)
    n = 200_000
    tx = np.asarray(txs, np.int32)[rng.integers(0, len(txs), n)]
    ri = rng.integers(0, len(rx), n).astype(np.int32)
    t = rng.uniform(0.0, 60.0, n)
    report = {}
    for scheme, sname in ((N.LPK_ITER_FIXED_POINT, "fixed-point"), (N.LPK_ITER_NEWTON, "newton")):
        res = {}
        for start, lname in ((N.LPK_START_LAG, "lag"), (N.LPK_START_GEOMETRIC, "geometric"),
                             (N.LPK_START_LEARNED, "learned")):
            te, it, err, _ = N.solve_converged_scene(ctx, tx, ri, rx, sc.epoch_unix, t, tol=1e-12, max_iter=12,
                                                     scheme=scheme, start=start, mlp=m)
            assert np.all(it > 0)
            res[lname] = (te, float(it.mean()), float(np.median(err)), float(np.max(err)))
        for lname in ("geometric", "learned"):
            assert np.max(np.abs(res[lname][0] - res["lag"][0])) <= 2e-12
        report[sname] = {k: {"mean_evals": v[1], "median_start_err_s": v[2], "max_start_err_s": v[3]}
                         for k, v in res.items()}
        assert res["learned"][1] < res["lag"][1]
        assert res["learned"][1] <= res["geometric"][1] + 1e-9
        assert res["learned"][2] < 0.1 * res["geometric"][2]
    print("converged solve, |residual| < 1e-12 s, 64 x 16 scene:", report)
    m.close()
