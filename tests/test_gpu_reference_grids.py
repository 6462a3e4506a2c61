"""GPU parity at the benched grid and the ensemble grids, against the reference solver itself.

The compiled reference (``oracle/_ref/<grid>/les_ref``, built from ``les_combustion_solver.c``
by ``oracle/build_ref.py``) runs live on the host cores beside the GPU solver, seed 1234:

* 256x128x128 / 800 eddies (the grid bench.py measures): states after 1 and 10 steps;
* 128x64x64 / 400 eddies and 96x48x48 / 300 eddies (the two ensemble grids): 10 steps.

The reference uses every host core (``OMP_NUM_THREADS``) with its inflow loop on one thread
(``LES_REF_SERIAL_BC=1``), so its three ``rand()`` draws per inlet cell come in the serial
(j, k) order that the GPU solver reproduces; only the order of its OpenMP sums depends on
the thread count, at rounding level.

Tolerances (the drop-in's parity bar), relative L2 per state field ||gpu - ref|| / ||ref||:
1e-10 after 1 step, 1e-8 after 10 steps; nu_t and |S| at the same bars.  The dt sequence
must agree to 1e-13 relative (it is taken from maxima of fields that agree to rounding).
The probe rows (les_combustion_solver.c:3403-3471, printed with %.6f / %.6e) must have the
same rows and agree to one unit of the last printed digit.  Observed errors are printed
(run with ``-s`` or ``-rP`` to see them).
"""
import os

import numpy as np
import pytest

from refcompare import compare_probes, read_probe_texts, rel

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
EXTRA = ["nu_t", "S_mag"]
TOL_1 = 1e-10
TOL_10 = 1e-8
TOL_DT = 1e-13


def _run_case(N, oracle_mod, grid, steps, keep, tmp_path):
    from lesgpu.config import preset
    if not oracle_mod.ref_available(grid):
        pytest.skip(f"compiled reference for {grid} not present (oracle/build_ref.py)")
    threads = os.cpu_count() or 1
    dumps, meta = oracle_mod.run_reference(
        grid, steps, seed=1234, dump_every=steps, threads=threads,
        env_extra={"LES_REF_SERIAL_BC": 1, "LES_REF_DUMP_FIRST": 1 if 1 in keep else 0})
    cfg = preset(grid, seed=1234)
    gdir = tmp_path / "gpu"
    gdir.mkdir()
    sol = N.Solver(cfg)
    sol.set_outputs(str(gdir), N.LES_OUT_PROBES)
    dts, states = [], {}
    for n in range(1, steps + 1):
        sol.step()
        dts.append(sol.last_dt)
        if n in keep:
            st = sol.state()
            for f in EXTRA:
                st[f] = sol.field(f)
            states[n] = st
    sol.flush()
    sol.close()
    ref_dt = np.array([t[1] for t in meta["times"]])
    assert len(ref_dt) == steps
    dt_err = float(np.max(np.abs(np.array(dts) - ref_dt) / ref_dt))
    print(f"\n[{grid}] reference on {threads} host threads; dt sequence max rel diff {dt_err:.3e}")
    assert dt_err <= TOL_DT, f"{grid}: dt differs by {dt_err:.3e}"
    for n in keep:
        tol = TOL_1 if n == 1 else TOL_10
        errs = {f: rel(states[n][f], dumps[n][f]) for f in STATE + EXTRA}
        k = max(errs, key=errs.get)
        print(f"[{grid}] step {n}: worst rel L2 {errs[k]:.3e} ({k}); "
              + ", ".join(f"{f} {errs[f]:.1e}" for f in STATE + EXTRA))
        assert errs[k] <= tol, f"{grid} step {n}: {k} rel L2 {errs[k]:.3e} > {tol}"
    pw = compare_probes(read_probe_texts(str(gdir)), meta["probes"])
    print(f"[{grid}] probe rows after {steps} steps: identical row sets, max |diff| {pw:.2e}")


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def test_benched_grid_256x128x128_matches_reference(N, oracle_mod, tmp_path):
    """The bench.py workload (4.19 M cells, 800 eddies): 1 and 10 steps."""
    _run_case(N, oracle_mod, "c2", 10, (1, 10), tmp_path)


@pytest.mark.parametrize("grid", ["e128", "e96"])
def test_ensemble_grids_match_reference(N, oracle_mod, grid, tmp_path):
    """The two grids of the batched ensemble: 1 and 10 steps."""
    _run_case(N, oracle_mod, grid, 10, (1, 10), tmp_path)
