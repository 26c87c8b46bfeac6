"""Surrogate pieces that need no GPU: the FP64 network oracle, features and
targets, the query draws and the C ABI's parameter count."""
from __future__ import annotations

import numpy as np
import pytest

import mlp_ref
from elasticscattering_b200 import _native as N
from elasticscattering_b200 import surrogate as S


def test_reference_backprop_matches_finite_differences():
    """The oracle's analytic gradient (rounding off) against central differences."""
    rng = np.random.default_rng(1)
    p = S.init_params(1, seed=3).astype(np.float64)
    x = rng.uniform(-1, 1, size=(6, 5))
    y = rng.uniform(-1, 1, size=(6, 2))
    _, g = mlp_ref.loss_and_grads(p, x, y, rounding=False)
    layers = [0]
    for k, n in zip(mlp_ref.DIMS[:-1], mlp_ref.DIMS[1:]):
        layers.append(layers[-1] + k * n + n)
    picks = [3, layers[1] - 1, layers[1] + 700, layers[2] + 12345, layers[4] + 5, layers[5] - 1, layers[5] - 300]
    h = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_ref.loss_and_grads(pp, x, y, rounding=False)[0] - mlp_ref.loss_and_grads(pm, x, y, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    # BF16 keeps 8 significant bits: the spacing above 1 is 2^-7
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3],
                 dtype=np.float32)
    r = mlp_ref.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                    # halfway between 1 and 1 + 2^-7: ties to the even significand
    assert r[2] == 1.0 + 2 ** -7          # above halfway rounds up
    assert r[3] == 1.0                    # below halfway rounds down
    assert r[4] == 1.0 + 2 ** -6          # halfway between 1 + 2^-7 (odd) and 1 + 2^-6 (even)
    assert r[5] == -2.5
    assert abs(r[6] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_param_count_agrees_with_the_library():
    assert mlp_ref.param_count() == 199426
    assert int(N.cuda_lib().es_mlp_param_count()) == mlp_ref.param_count()
    assert S.init_params(4, 0).size == 4 * mlp_ref.param_count()


def test_features_and_targets():
    q = S.sample_queries(2000, seed=5)
    assert (q[:, 0] >= 0.5).all() and (q[:, 0] <= 50).all()
    assert (q[:, 2] >= 5e14).all() and (q[:, 2] <= 2e16).all()
    assert (q[:, 4] >= 1e-13).all() and (q[:, 4] <= 1e-11).all()
    f = S.features(q)
    assert f.dtype == np.float32 and f.shape == (2000, 5)
    assert f[:, [0, 1, 2, 4]].min() >= -1.0001 and f[:, [0, 1, 2, 4]].max() <= 1.0001
    sigma = 0.7 * S.sigma0(q[:, 4])[:, None] * S.drude(q)
    t = S.targets(q, sigma)
    assert np.allclose(t, np.log(0.7), atol=1e-6)
    back = S.untarget(q, t)
    assert np.allclose(back, sigma, rtol=2e-6)
    with pytest.raises(ValueError):
        S.targets(q[:1], -sigma[:1])
    # the Drude scale is linear in tau
    assert S.sigma0(2e-12) == pytest.approx(2 * S.sigma0(1e-12))


def test_training_draw_stays_in_the_config4_ranges():
    q = S.training_queries(4000, seed=3)
    assert q.shape == (4000, 5)
    assert (q[:, 0] >= S.B_RANGE[0]).all() and (q[:, 0] <= S.B_RANGE[1]).all()
    assert (q[:, 1] >= S.T_RANGE[0]).all() and (q[:, 1] <= S.T_RANGE[1]).all()
    assert (q[:, 2] >= S.N_RANGE[0]).all() and (q[:, 2] <= S.N_RANGE[1]).all()
    assert (q[:, 4] >= S.TAU_RANGE[0]).all() and (q[:, 4] <= S.TAU_RANGE[1]).all()
    hard = q[2000:]
    in_hard = ((hard[:, 0] <= S.HARD_B[1]) | (hard[:, 4] >= S.HARD_TAU[0]) | (hard[:, 1] <= S.HARD_T[1]))
    assert in_hard.all()
    assert np.array_equal(S.training_queries(100, seed=3, hard_fraction=0.0), S.sample_queries(100, seed=3))


def test_query_map_reproduces_features_and_untarget():
    """The map es_mlp_query evaluates on the device, applied here in numpy with
    the device's formula, gives features() bit for bit and untarget() to
    rounding."""
    m = S.query_map()
    q = S.sample_queries(2000, seed=3)
    f = np.empty((len(q), 5))
    for k in range(5):
        g = np.log(q[:, k]) if m.log_scale[k] else q[:, k]
        f[:, k] = 2.0 * (g - m.g_lo[k]) / (m.g_hi[k] - m.g_lo[k]) - 1.0
    assert np.array_equal(f.astype(np.float32), S.features(q))
    t = np.random.default_rng(4).normal(size=(3, len(q), 2)).astype(np.float32)
    wt = m.w_per_b * q[:, 0] * q[:, 4]
    shape = np.stack([1.0 / (1.0 + wt * wt), wt / (1.0 + wt * wt)], axis=1)
    dev = np.exp(t.astype(np.float64)) * (m.sigma0_per_tau * q[:, 4])[:, None] * shape
    assert np.allclose(dev, S.untarget(q, t), rtol=1e-14, atol=0)
