"""The learned warm start of the converged emission solve: tensor-core
forward and gradient kernels against the CPU restatement, the converged
solver against the oracle's 80-bit solve, and what the trained network
gains over starting where the reference starts (t - 70 ms)."""
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
FORWARD_ATOL = 2e-3  # outputs are O(1)
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
    x = rng.normal(size=(1000, M.N_F)).astype(np.float32)  # not a multiple of the 16-row warp tile
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
    for name, a, b in (("W1", M.OFF_W1, M.OFF_B1), ("b1", M.OFF_B1, M.OFF_W2), ("W2", M.OFF_W2, M.OFF_B2),
                       ("b2", M.OFF_B2, M.OFF_W3), ("w3", M.OFF_W3, M.OFF_B3), ("b3", M.OFF_B3, M.N_PARAMS)):
        err = np.linalg.norm(g[a:b] - gr[a:b]) / max(np.linalg.norm(gr[a:b]), 1e-30)
        assert err <= GRAD_RTOL, (name, n, err)
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


def test_learned_start_cuts_iterations(ctx, dual):
    sc, prep, rx, epoch = dual
    rng = np.random.default_rng(11)
    t = np.sort(rng.uniform(0.0, 120.0, 20000))
    report = {}
    for tx, label in ((0, "LEO 437 MHz"), (1, "GPS PRN 1")):
        m = N.Mlp(ctx, seed=5)
        curve = m.fit(tx, rx, epoch, 0.0, 120.0, n_train=1 << 18, steps=1500, batch=4096, lr=3e-3, seed=9)
        assert curve[-50:].mean() < 0.02 * curve[:20].mean(), (curve[:5], curve[-5:])
        out = {}
        for scheme, sname in ((N.LPK_ITER_FIXED_POINT, "fixed-point"), (N.LPK_ITER_NEWTON, "newton")):
            res = {}
            for start, lname in ((N.LPK_START_LAG, "lag"), (N.LPK_START_GEOMETRIC, "geometric"),
                                 (N.LPK_START_LEARNED, "learned")):
                te, it, err = N.solve_converged(ctx, tx, rx, epoch, t, tol=1e-13, max_iter=12, scheme=scheme,
                                                start=start, mlp=m)
                assert np.all(it > 0)
                res[lname] = (te, float(it.mean()), float(np.median(err)), float(np.max(err)))
            # every start converges to the same emission times
            for lname in ("geometric", "learned"):
                assert np.max(np.abs(res[lname][0] - res["lag"][0])) <= 2e-13
            out[sname] = {k: {"mean_evals": v[1], "median_start_err_s": v[2], "max_start_err_s": v[3]}
                          for k, v in res.items()}
            assert res["learned"][1] < res["lag"][1]
            assert res["learned"][2] < 0.1 * res["geometric"][2]
        assert out["fixed-point"]["learned"]["mean_evals"] < out["fixed-point"]["geometric"]["mean_evals"]
        report[label] = out
        m.close()
    print("converged solve, tol 1e-13 s:", report)
