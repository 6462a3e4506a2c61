"""Profile statistics of the probe rows against the reference's own post-processing
(tests/golden/stats_ref.npz, made by tests/golden/make_stats_golden.py from
bayesian_optimizer.py and analysis.py run on a seeded synthetic probe file)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

TOL = 1e-12


@pytest.fixture(scope="module")
def golden(tmp_path_factory):
    z = np.load(os.path.join(GOLDEN, "stats_ref.npz"))
    d = tmp_path_factory.mktemp("probe")
    path = d / "probe_data_flame_region_loc0.csv"
    path.write_bytes(z["csv_text"].tobytes())
    from lesgpu import stats
    return z, stats.read_probe_csv(str(path)), stats


def close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(b)
    np.testing.assert_allclose(a[ok], b[ok], rtol=TOL, atol=TOL * np.abs(b[ok]).max())


def test_uv_vs_g_matches_bayesian_optimizer(golden):
    z, rows, stats = golden
    g, s = stats.uv_vs_g(rows, 20)
    close(g, z["uv_G_centers"])
    close(s, z["uv_stress"])
    g, s = stats.uv_vs_g(rows, 37)
    close(g, z["uv37_G_centers"])
    close(s, z["uv37_stress"])


def test_flame_profile_matches_analysis(golden):
    z, rows, stats = golden
    p = stats.flame_profile(rows)
    for k in ("re_uu", "re_vv", "re_ww", "re_uv", "G"):
        close(p["bin_center"], z[f"flame_profile.{k}.x"])
        close(p[k], z[f"flame_profile.{k}.y"])


def test_stress_vs_g_matches_analysis(golden):
    z, rows, stats = golden
    p = stats.stress_vs_g(rows)
    for k in ("uu_cond", "vv_cond", "uv_cond"):
        close(p["G_center"], z[f"stress_vs_G.{k}.x"])
        close(p[k], z[f"stress_vs_G.{k}.y"])


def test_compare_profiles_zero_for_identical_and_detects_change(golden):
    z, rows, stats = golden
    e = stats.compare_profiles(rows, rows)
    assert e and all(v == 0.0 for v in e.values())
    pert = dict(rows)
    pert["u"] = rows["u"] * (1 + 1e-3)
    e = stats.compare_profiles(pert, rows)
    assert 5e-4 < e["flame_profile.mean_u"] < 2e-3
    assert e["stress_vs_G.uu_cond"] > 1e-3


def test_conditional_pdfs_normalised(golden):
    z, rows, stats = golden
    eu, ev = np.linspace(0, 14, 57), np.linspace(-3, 3, 49)
    p = stats.conditional_pdfs(rows, eu, ev)
    for k, e in (("u_unburnt", eu), ("u_burnt", eu), ("v_unburnt", ev), ("v_burnt", ev)):
        assert abs((p[k] * np.diff(e)).sum() - 1.0) < 1e-12
