"""The optimiser restated from bayesian_optimizer.py against the reference's own functions
(tests/golden/stats_ref.npz, made by tests/golden/make_stats_golden.py): the experimental fit,
the profile smoothing and score, the GP expected improvement and the next proposal."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def z():
    return np.load(os.path.join(GOLDEN, "stats_ref.npz"))


@pytest.fixture(scope="module")
def O():
    from lesgpu import optimizer
    return optimizer


def test_experimental_fit(z, O):
    np.testing.assert_allclose(O.experimental_reynolds_stress(z["exp_G"]), z["exp_val"], rtol=1e-15, atol=0)


def test_smoothing_and_score(z, O):
    G = z["prof_G"]
    for q in range(3):
        p = z["prof_val"][q]
        g, v = O.smooth_profile(G[~np.isnan(p)], p[~np.isnan(p)])
        np.testing.assert_allclose(g, z["smooth_G"][q], rtol=1e-14)
        np.testing.assert_allclose(v, z["smooth_val"][q], rtol=1e-12, atol=1e-17)
    got = np.array([O.compute_score(G, p) for p in z["prof_val"]])
    np.testing.assert_allclose(got, z["prof_score"], rtol=1e-10)
    assert got.max() == 1e6 or (z["prof_score"] < 1e6).all()
    np.testing.assert_allclose(O.compute_score(z["uv_G_centers"], z["uv_stress"]), z["uv_score"][0], rtol=1e-10)


def test_expected_improvement_and_proposal(z, O):
    opt = O.BayesianOptimizer()
    opt.X_obs = [list(map(float, x)) for x in z["ei_X"]]
    opt.y_obs = list(map(float, z["ei_y"]))
    np.random.seed(6)
    ei = opt.expected_improvement(z["ei_cand"])
    np.testing.assert_allclose(ei, z["ei"], rtol=1e-7, atol=1e-12)
    np.random.seed(9)
    nxt = opt.suggest_next(n_candidates=500)
    np.testing.assert_allclose([nxt[k] for k in opt.param_names], z["next"], rtol=1e-12)


def test_batch_proposals_are_distinct_and_in_bounds(O):
    opt = O.BayesianOptimizer(rng=np.random.default_rng(3))
    rng = np.random.default_rng(4)
    for _ in range(6):
        x = {k: rng.uniform(*O.PARAM_BOUNDS[k]) for k in opt.param_names}
        opt.register_result(x, float(rng.random()))
    batch = opt.suggest_batch(4, n_candidates=400)
    assert len(batch) == 4
    arr = np.array([[b[k] for k in opt.param_names] for b in batch])
    assert len({tuple(r) for r in arr.round(12)}) == 4
    for k, (lo, hi) in O.PARAM_BOUNDS.items():
        col = arr[:, opt.param_names.index(k)]
        assert (col >= lo).all() and (col <= hi).all()
    assert len(opt.y_obs) == 6          # pseudo-observations are not kept


def test_config_mapping(O):
    from lesgpu.config import preset
    base = preset("tiny")
    p = {k: 0.5 * (lo + hi) for k, (lo, hi) in O.PARAM_BOUNDS.items()}
    c = O.config_for(base, p)
    assert c.accel_strength == p["FLAME_ACCEL_STRENGTH"] and c.cs_burnt == p["CS_BURNT"]
    assert c.cs_flame_boost == p["CS_FLAME_BOOST"] and c.accel_center == p["FLAME_ACCEL_CENTER"]
    assert (c.nx, c.ny, c.nz) == (base.nx, base.ny, base.nz)
