"""The CPU restatement of the warm-start network (oracle/mlp_ref.py): its
bfloat16 rounding and its gradient, before it is used to check the
tensor-core kernels."""
import numpy as np

from oracle import mlp_ref as M


def test_bf16_rounds_to_nearest_even():
    one = 1.0
    assert M.bf16([one])[0] == 1.0
    assert M.bf16([1.0 + 2.0 ** -8])[0] == 1.0                       # tie -> even (1.0)
    assert M.bf16([1.0 + 3 * 2.0 ** -8])[0] == 1.0 + 2.0 ** -6      # tie -> even (k = 2)
    assert M.bf16([1.0 + 2.0 ** -8 + 2.0 ** -20])[0] == 1.0 + 2.0 ** -7
    assert M.bf16([-2.5])[0] == -2.5
    assert M.bf16([3.0e38])[0] > 2.9e38


def _random_params(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.4, 0.4, M.N_PARAMS)
    return p


def test_unquantised_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _random_params(2)
    x = rng.normal(size=(37, M.N_F))
    t = rng.normal(size=37)
    _, g = M.loss_grad(p, x, t, quantize=False)
    idx = np.r_[rng.choice(M.N_PARAMS, 60, replace=False), M.OFF_B4, M.OFF_W1, M.OFF_W2 + 5, M.OFF_W3 + 7,
                M.OFF_W4 + 3]
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_grad(pp, x, t, quantize=False)[0] - M.loss_grad(pm, x, t, quantize=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_quantised_gradient_stays_close_to_exact():
    rng = np.random.default_rng(3)
    p = _random_params(4)
    x = rng.normal(size=(256, M.N_F))
    t = rng.normal(size=256)
    _, gq = M.loss_grad(p, x, t)
    _, g = M.loss_grad(p, x, t, quantize=False)
    assert np.linalg.norm(gq - g) <= 0.05 * np.linalg.norm(g)


def test_orbit_state_velocity_is_the_derivative():
    orbit = (7.0e6, 51.6, 100.0, 270.0)
    e = np.array([0.0, 13.7, 59.9])
    h = 1e-3
    p0, v0 = M.orbit_state(orbit, e)
    pp, _ = M.orbit_state(orbit, e + h)
    pm, _ = M.orbit_state(orbit, e - h)
    assert np.max(np.abs((pp - pm) / (2 * h) - v0)) < 1e-3  # m/s
    assert np.allclose(np.linalg.norm(p0, axis=1), 7.0e6)
