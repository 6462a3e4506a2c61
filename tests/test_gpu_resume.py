"""Resume on the GPU (les_solver_finish / les_solver_resume).

* LES_RESUME_REFERENCE against the reference's own auto-resume: the compiled reference runs
  20 steps of the 64x32x32 case, exits (saving "step 0", les_combustion_solver.c:4623), and is
  started again in the same directory, which resumes from restart_info.txt with its defects
  (rand() re-seeded and vortices redrawn, :4193; the start-up attribute map without setting(),
  :4123-4136; nu/alpha maxima 0) for 10 more steps.  The GPU solver does the same through
  les_solver_finish / les_solver_resume; the state after the resumed steps must agree at the
  10-step parity bar (relative L2 1e-8 per field), the dt sequence to 1e-13.
* LES_RESUME_FIXED: 20 steps, finish, resume in a new solver, 10 steps -- bit-identical to
  30 uninterrupted steps (state, dt, vortices, rand() draws).
"""
import os

import numpy as np
import pytest

from refcompare import rel

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def test_reference_mode_resume_matches_the_reference_resume(N, oracle_mod, tmp_path):
    from lesgpu.config import preset
    if not oracle_mod.ref_available("c1"):
        pytest.skip("compiled reference for c1 not present")
    threads = os.cpu_count() or 1
    rdir = str(tmp_path / "ref")
    env = {"LES_REF_SERIAL_BC": 1}
    oracle_mod.run_reference("c1", 20, seed=1234, dump_every=20, threads=threads, env_extra=env, keep_dir=rdir)
    with open(os.path.join(rdir, "restart_info.txt")) as f:
        assert f.read() == "BINARY\n0\n"
    dumps, meta = oracle_mod.run_reference("c1", 10, seed=1234, dump_every=10, threads=threads, env_extra=env,
                                           keep_dir=rdir, resume=True)
    assert "AUTO-RESUME" in meta["stdout"]
    cfg = preset("c1", seed=1234)
    gdir = str(tmp_path / "gpu")
    os.makedirs(gdir)
    a = N.Solver(cfg)
    a.step(20)
    a.finish(gdir, N.RESUME_REFERENCE)
    a.close()
    b = N.Solver(cfg)
    assert b.resume(gdir, N.RESUME_REFERENCE) == 0
    dts = []
    for _ in range(10):
        b.step()
        dts.append(b.last_dt)
    st = b.state()
    attr = b.attribute()
    b.close()
    assert (attr[1:-1, 0, 1:-1] == 4).all()
    ref_dt = np.array([t[1] for t in meta["times"]])
    dt_err = float(np.max(np.abs(np.array(dts) - ref_dt) / ref_dt))
    errs = {f: rel(st[f], dumps[10][f]) for f in STATE}
    k = max(errs, key=errs.get)
    print(f"\n[resume, reference mode] dt max rel diff {dt_err:.2e}; state worst rel L2 {errs[k]:.2e} ({k})")
    assert dt_err <= 1e-13
    assert errs[k] <= 1e-8, errs


def test_fixed_mode_resume_is_bit_identical(N, tmp_path):
    from lesgpu.config import preset
    cfg = preset("c1", seed=77)
    a = N.Solver(cfg)
    a.step(20)
    a.finish(str(tmp_path), N.RESUME_FIXED)
    a.step(10)
    b = N.Solver(cfg)
    assert b.resume(str(tmp_path), N.RESUME_FIXED) == 20
    b.step(10)
    assert a.t_loop == b.t_loop == 30
    assert a.last_dt == b.last_dt
    assert a.rng_draws == b.rng_draws
    np.testing.assert_array_equal(a.vortices(), b.vortices())
    sa, sb = a.state(), b.state()
    for f in STATE:
        np.testing.assert_array_equal(sa[f], sb[f], err_msg=f)
    a.close()
    b.close()
