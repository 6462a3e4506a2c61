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


def test_from_moments_matches_the_row_statistics():
    """The device keeps moment sums per bin (lesgpu_pstat_*); stats.from_moments must turn
    them into the same statistics as the row-based functions.  The moments are formed here
    with numpy from seeded rows, binned with the edges' own semantics."""
    from lesgpu import stats
    rng = np.random.default_rng(11)
    n = 20000
    G = rng.uniform(0.0, 1.0, n)
    G[:300] = 0.0
    G[300:600] = 1.0
    G[600:700] = 0.5
    rows = {"y_relative": rng.uniform(-0.03, 0.03, n), "u": 5.0 + rng.normal(0, 0.8, n),
            "v": rng.normal(0, 0.5, n), "w": rng.normal(0, 0.4, n), "G": G}
    e = stats.default_edges(0.064, 5.0)
    u, v, w = rows["u"], rows["v"], rows["w"]
    ny, nrc, nho, npdf = (len(e[k]) - 1 for k in ("y_mm", "g_rc", "g_ho", "u"))
    sums = [len(u), u.sum(), v.sum(), w.sum()]
    by = stats._right_closed_bins(rows["y_relative"] * 1000, e["y_mm"])
    for b in range(ny):
        m = by == b
        sums += [m.sum(), u[m].sum(), v[m].sum(), w[m].sum(), G[m].sum(), (u[m] * u[m]).sum(), (v[m] * v[m]).sum(),
                 (w[m] * w[m]).sum(), (u[m] * v[m]).sum()]
    bg = stats._right_closed_bins(G, e["g_rc"])
    for b in range(nrc):
        m = bg == b
        sums += [m.sum(), u[m].sum(), v[m].sum(), w[m].sum(), (u[m] * u[m]).sum(), (v[m] * v[m]).sum(),
                 (u[m] * v[m]).sum()]
    for b in range(nho):
        m = (G >= e["g_ho"][b]) & (G < e["g_ho"][b + 1])
        sums += [m.sum(), u[m].sum(), v[m].sum(), (u[m] * v[m]).sum()]
    for k, burnt in (("u", False), ("v", False), ("u", True), ("v", True)):
        m = (G >= 0.5) if burnt else (G < 0.5)
        h, _ = np.histogram(rows[k][m], bins=e[k])
        sums += list(h)
    got = stats.from_moments(np.array(sums, dtype=np.float64), e)
    fp = stats.flame_profile(rows, e["y_mm"])
    for k in ("bin_center", "u", "v", "w", "G", "re_uu", "re_vv", "re_ww", "re_uv"):
        np.testing.assert_allclose(got["flame_profile"][k], fp[k], rtol=1e-9, atol=1e-12, err_msg=k)
    sg = stats.stress_vs_g(rows)
    for k in ("uu_cond", "vv_cond", "uv_cond", "u_mean", "v_mean", "w_mean", "G_center"):
        np.testing.assert_allclose(got["stress_vs_g"][k], sg[k], rtol=1e-9, atol=1e-12, err_msg=k)
    c, st = stats.uv_vs_g(rows)
    np.testing.assert_allclose(got["uv_vs_g"][0], c, rtol=0, atol=0)
    np.testing.assert_allclose(got["uv_vs_g"][1], st, rtol=1e-9, atol=1e-12)
    pd = stats.conditional_pdfs(rows, e["u"], e["v"])
    for k in pd:
        np.testing.assert_allclose(got["conditional_pdfs"][k], pd[k], rtol=1e-12, err_msg=k)


def test_probe_rows_follow_the_reference_writer():
    """stats.probe_rows (rows at full precision from probe lines) keeps the reference's rule:
    the lower G = 0.5 crossing, interpolated, and no rows when y_flame <= 0."""
    from lesgpu import stats
    ny, dy = 8, 0.002
    lines = np.zeros((2, 2, ny, 6))
    lines[0, 0, :, 3] = [1, 1, 1, 0.8, 0.3, 0, 0, 0]     # crossing between j = 3 and 4
    lines[0, 1, :, 3] = [0.2, 0.2, 0.7, 1, 1, 1, 1, 1]   # between j = 1 and 2
    lines[1, 0, :, 3] = 0.7                              # none
    lines[1, 1, :, 3] = [0.5, 0.5, 0, 0, 0, 0, 0, 0]     # at j = 0: y_flame = 0, no rows
    lines[..., 0] = np.arange(ny)
    r = stats.probe_rows(lines, 10, dy, np.array([0.01, 0.02]))
    assert len(r["u"]) == 2 * ny
    yf0 = 3 * dy + (0.5 - 0.8) / (0.3 - 0.8) * dy
    yf1 = 1 * dy + (0.5 - 0.2) / (0.7 - 0.2) * dy
    np.testing.assert_array_equal(r["y_flame"], np.r_[np.full(ny, yf0), np.full(ny, yf1)])
    np.testing.assert_array_equal(r["timestep"], np.full(2 * ny, 10.0))
    np.testing.assert_array_equal(r["u"], np.r_[np.arange(ny), np.arange(ny)])
