"""Profile statistics accumulated on the device (lesgpu_pstat_*, les_solver_pstat_*), no probe
files: a device-loop run of the 64x32x32 case in several chunks (the last one partial) with
the statistics on, against the row-based statistics of lesgpu/stats.py (pinned to the
reference's post-processing by tests/test_stats.py) computed from the same rows at full
precision.  The rows come from a host-driven run of the same case (bit-identical to the
device loop, tests/test_gpu_parity.py) through lesgpu_probe_lines every step, with the
reference writer's y_flame rule (les_combustion_solver.c:3419-3466, stats.probe_rows).

Bin counts must agree exactly; means and Reynolds stresses to 1e-9 relative (raw moments
against two-pass fluctuations), the PDFs to 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def test_device_statistics_match_the_row_statistics(N):
    from lesgpu import stats
    from lesgpu.config import preset
    cfg = preset("c1", seed=99)
    steps = 150
    a = N.Solver(cfg)
    edges = a.pstat_begin()
    a.run_device(steps, chunk=40)
    got = a.profile_stats()
    sums = a.pstat_read()
    a.close()
    b = N.Solver(cfg)
    dx, dy = cfg.lx / cfg.nx, cfg.ly / cfg.ny
    xs = np.array([0.010, 0.015, 0.020, 0.025, 0.030, 0.035, 0.040])
    st = [int(x / dx) for x in xs]
    keep = [q for q, i in enumerate(st) if 0 < i < cfg.nx - 1]
    lines = []
    for _ in range(steps):
        b.step()
        lines.append(b.ctx.probe_lines([st[q] for q in keep], cfg.nz // 2))
    b.close()
    rows = stats.probe_rows(np.array(lines), 0, dy, xs[keep])
    assert len(rows["u"]) > 5000
    assert sums[0] == len(rows["u"])
    fp = stats.flame_profile(rows, edges["y_mm"])
    print(f"\n[pstat c1 x {steps}] {len(rows['u'])} rows; "
          f"re_uu max rel diff {np.max(np.abs(got['flame_profile']['re_uu'] - fp['re_uu']) / np.abs(fp['re_uu'])):.2e}")
    np.testing.assert_array_equal(got["flame_profile"]["bin_center"], fp["bin_center"])
    for k in ("u", "v", "w", "G", "re_uu", "re_vv", "re_ww", "re_uv"):
        np.testing.assert_allclose(got["flame_profile"][k], fp[k], rtol=1e-9, atol=1e-13, err_msg=k)
    sg = stats.stress_vs_g(rows)
    np.testing.assert_array_equal(got["stress_vs_g"]["G_center"], sg["G_center"])
    for k in ("uu_cond", "vv_cond", "uv_cond", "u_mean", "v_mean", "w_mean"):
        np.testing.assert_allclose(got["stress_vs_g"][k], sg[k], rtol=1e-9, atol=1e-13, err_msg=k)
    _, uv = stats.uv_vs_g(rows)
    np.testing.assert_array_equal(np.isnan(got["uv_vs_g"][1]), np.isnan(uv))
    np.testing.assert_allclose(got["uv_vs_g"][1], uv, rtol=1e-9, atol=1e-13)
    pd = stats.conditional_pdfs(rows, edges["u"], edges["v"])
    for k in pd:
        np.testing.assert_allclose(got["conditional_pdfs"][k], pd[k], rtol=1e-12, atol=0, err_msg=k)
