"""Profile statistics over long runs: the quantities the reference's post-processing and its
Bayesian optimiser draw from the probe files (les_combustion_solver.c:3403-3471 rows,
statistics of analysis.py:112-154, :215-257 and bayesian_optimizer.py:71-117, restated in
lesgpu/stats.py and pinned to the reference's own functions by tests/test_stats.py).

* Plain FP64 form against the reference solver itself, 64x32x32 / 200 eddies, 600 steps
  (crossing the t_loop = 500 switch to the WENO5 flame-front gradient).  The reference runs
  live on the host cores with its inflow loop on one thread (LES_REF_SERIAL_BC=1, so its
  rand() draws come in the serial order).  Both runs print the probe rows with %.6f, so the
  profiles can agree no better than the printed digits: stated tolerance 1e-6 relative L2
  per profile; the final state at the 10-step bar, 1e-8 relative L2 per field.
* FP32-bulk precision form against the FP64 form, 128x64x64 / 400 eddies (an ensemble grid),
  500 steps: the mean axial velocity, the Reynolds stresses u'u', v'v', w'w', u'v' against
  the distance from the flame front and against G, <u'v'> in the optimiser's 20 G bins, and
  the conditional velocity PDFs, each within 1e-3 relative L2 of the FP64 run -- the
  precision form's stated bound.

Observed errors are printed (run with -s or -rP).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
TOL_PROFILE_FP64 = 1e-6
TOL_STATE_FP64 = 1e-8
TOL_PROFILE_FP32 = 1e-3


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _pool_texts(texts):
    import io
    from lesgpu import stats
    parts = []
    for n in sorted(texts):
        body = texts[n].split("\n", 1)[1] if "\n" in texts[n] else ""
        if body.strip():
            d = np.loadtxt(io.StringIO(body), delimiter=",", ndmin=2)
            parts.append({c: d[:, q] for q, c in enumerate(stats.COLUMNS)})
    return {c: np.concatenate([p[c] for p in parts]) for c in stats.COLUMNS}


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def test_fp64_long_run_profiles_match_reference(N, oracle_mod, tmp_path):
    from lesgpu import precision, stats
    from lesgpu.config import preset
    if not oracle_mod.ref_available("c1"):
        pytest.skip("compiled reference for c1 not present (oracle/build_ref.py)")
    steps = 600
    dumps, meta = oracle_mod.run_reference("c1", steps, seed=1234, dump_every=steps, threads=os.cpu_count() or 1,
                                           env_extra={"LES_REF_SERIAL_BC": 1})
    cfg = preset("c1", seed=1234)
    d = tmp_path / "gpu"
    d.mkdir()
    sol = N.Solver(cfg)
    sol.set_outputs(str(d), N.LES_OUT_PROBES)
    sol.run_device(steps, chunk=100)
    st = sol.state()
    sol.close()
    serr = {f: rel(st[f], dumps[steps][f]) for f in STATE}
    kw = max(serr, key=serr.get)
    print(f"\n[c1 x {steps}] final state worst rel L2 {serr[kw]:.3e} ({kw})")
    rows_gpu = precision._pool(str(d))
    rows_ref = _pool_texts(meta["probes"])
    assert len(rows_gpu["u"]) == len(rows_ref["u"]) > 1000
    errs = stats.compare_profiles(rows_gpu, rows_ref)
    print(f"[c1 x {steps}] {len(rows_ref['u'])} probe rows; profile rel L2: "
          + ", ".join(f"{k} {v:.1e}" for k, v in sorted(errs.items())))
    assert serr[kw] <= TOL_STATE_FP64, f"state {kw}: {serr[kw]:.3e}"
    bad = {k: v for k, v in errs.items() if not v <= TOL_PROFILE_FP64}
    assert not bad, bad


def test_fp32_profiles_within_bound_of_fp64(N, tmp_path):
    from lesgpu import precision
    from lesgpu.config import preset
    steps = 500
    out = precision.compare(preset("e128"), steps, workdir=str(tmp_path), chunk=100, floor=())
    errs = out["profiles_fp32"]
    print(f"\n[e128 x {steps}] rows fp64 {out['rows_fp64']} fp32 {out['rows_fp32']}; FP32 vs FP64 profile rel L2: "
          + ", ".join(f"{k} {v:.1e}" for k, v in sorted(errs.items())))
    print(f"[e128 x {steps}] state rel L2: " + ", ".join(f"{k} {v:.1e}" for k, v in out["state_rel_l2_fp32"].items()))
    assert out["rows_fp64"] > 1000
    wanted = ["flame_profile.mean_u", "flame_profile.re_uu", "flame_profile.re_vv", "flame_profile.re_ww",
              "flame_profile.re_uv", "stress_vs_G.u_mean", "stress_vs_G.uu_cond", "stress_vs_G.vv_cond",
              "stress_vs_G.uv_cond", "uv_vs_G", "pdf.u_unburnt", "pdf.v_unburnt", "pdf.u_burnt", "pdf.v_burnt"]
    missing = [k for k in wanted if k not in errs]
    assert not missing, missing
    bad = {k: errs[k] for k in wanted if not errs[k] <= TOL_PROFILE_FP32}
    assert not bad, bad
