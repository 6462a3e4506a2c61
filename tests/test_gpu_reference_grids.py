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

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
EXTRA = ["nu_t", "S_mag"]
TOL_1 = 1e-10
TOL_10 = 1e-8
TOL_DT = 1e-13


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _parse_probe(text):
    rows = [ln.split(",") for ln in text.splitlines()[1:] if ln.strip()]
    return np.array([[float(x) for x in r] for r in rows]).reshape(-1, 11)


def _compare_probes(gpu_dir, ref_probes):
    worst = 0.0
    for n in range(7):
        path = os.path.join(gpu_dir, f"probe_data_flame_region_loc{n}.csv")
        ref_txt = ref_probes.get(n)
        if ref_txt is None:
            assert not os.path.exists(path), f"station {n}: GPU wrote rows the reference did not"
            continue
        with open(path) as f:
            gpu_txt = f.read()
        a, b = _parse_probe(gpu_txt), _parse_probe(ref_txt)
        assert a.shape == b.shape, f"station {n}: {a.shape[0]} rows against the reference's {b.shape[0]}"
        # timestep, x, y_flame, y, y_rel, u, v, w, G at %.6f: one unit of the 6th decimal
        d_fixed = np.abs(a[:, :9] - b[:, :9]).max(initial=0.0)
        assert d_fixed <= 1.01e-6, f"station {n}: fixed-point columns differ by {d_fixed:.3e}"
        # nu_t, |S| at %.6e: one unit of the 7th significant digit
        scale = np.maximum(np.abs(b[:, 9:]), 1e-300)
        d_exp = (np.abs(a[:, 9:] - b[:, 9:]) / scale).max(initial=0.0)
        assert d_exp <= 1.01e-6, f"station {n}: nu_t/S_mag differ by {d_exp:.3e} relative"
        worst = max(worst, d_fixed)
    return worst


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
    pw = _compare_probes(str(gdir), meta["probes"])
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
