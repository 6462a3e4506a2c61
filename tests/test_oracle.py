"""The oracle restatement is pinned to the reference solver itself.

* against the golden fixtures (states written by the compiled reference, tests/golden):
  bit-identical after every stored step, identical dt sequence;
* against the compiled reference live, when oracle/_ref exists on this machine
  (including the stage-1 RHS intermediates);
* the monitor line and the probe extraction rules against the reference's outputs.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4", "nu_t", "S_mag"]


def _golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


@pytest.mark.parametrize("case", ["tiny_s10", "tiny_w495", "small_s12"])
def test_oracle_matches_reference_fixtures(oracle_mod, case):
    from lesgpu.config import preset
    g = _golden(case)
    cfg = preset(str(g["config"]), seed=int(g["seed"]))
    orc = oracle_mod.Oracle(cfg.as_dict(), start_step=int(g["start"]))
    keep = set(int(x) for x in g["steps"])
    for n in range(1, len(g["dt"]) + 1):
        orc.step()
        assert orc.dt == g["dt"][n - 1], f"dt differs at step {n}"
        if n in keep:
            for f in STATE:
                np.testing.assert_array_equal(orc.field(f), g[f"s{n}_{f}"], err_msg=f"{case} step {n} field {f}")
    orc.close()


def test_monitor_line_format(oracle_mod):
    """write_monitor_log's row (les_combustion_solver.c:3915-3916) from the initial state,
    with the reference's serial mass sum, equals the reference's first monitor row."""
    from lesgpu.config import preset
    g = _golden("tiny_s10")
    cfg = preset("tiny")
    orc = oracle_mod.Oracle(cfg.as_dict())
    orc.step()
    st = orc.state()
    dx, dy, dz = cfg.lx / cfg.nx, cfg.ly / cfg.ny, cfg.lz / cfg.nz
    terms = ((st["rho"].ravel() * dx) * dy) * dz
    mass = np.cumsum(terms)[-1]
    row = "%d,%.6e,%.6e,%.2f,%.2f,%.4f,%.4f,%.2e" % (0, orc.dt, mass, st["T"].min(), st["T"].max(),
                                                    st["G"].min(), st["G"].max(), st["Y0"].min())
    mon = bytes(g["monitor"]).decode().splitlines()
    assert mon[0] == "step,dt,total_mass,min_T,max_T,min_G,max_G,min_Y_C3H8"
    assert mon[1] == row
    orc.close()


def test_oracle_matches_compiled_reference_live(oracle_mod):
    if not oracle_mod.ref_available("small"):
        pytest.skip("compiled reference not present (oracle/_ref is built where the reference source exists)")
    from lesgpu.config import preset
    cfg = preset("small", seed=4321)
    dumps, meta = oracle_mod.run_reference("small", 4, seed=4321, dump_every=1, rhs_dump_step=0)
    orc = oracle_mod.Oracle(cfg.as_dict())
    orc.rhs_only(0)
    for k, v in meta["rhs1"].items():
        np.testing.assert_array_equal(orc.field(k), v, err_msg=f"stage-1 intermediate {k}")
    orc.close()
    orc = oracle_mod.Oracle(cfg.as_dict())
    for n in range(1, 5):
        orc.step()
        assert orc.dt == dumps[n]["dt"]
        for f in STATE:
            np.testing.assert_array_equal(orc.field(f), dumps[n][f], err_msg=f"step {n} field {f}")
    orc.close()


def test_oracle_varied_constants_live(oracle_mod):
    """An ensemble member's constants (SGS constant, forcing amplitude, nudging coefficient)
    take the same path through the reference and the oracle."""
    if not oracle_mod.ref_available("tiny"):
        pytest.skip("compiled reference not present")
    from lesgpu.config import preset
    over = dict(cs_unburned=0.19, accel_strength=3.1, relax=1234.5)
    env = {"LES_REF_CS_UNBURNED": repr(over["cs_unburned"]), "LES_REF_ACCEL_STRENGTH": repr(over["accel_strength"]),
           "LES_REF_RELAX": repr(over["relax"])}
    dumps, _ = oracle_mod.run_reference("tiny", 3, seed=99, dump_every=3, env_extra=env)
    orc = oracle_mod.Oracle(preset("tiny", seed=99, **over).as_dict())
    orc.step(3)
    for f in STATE:
        np.testing.assert_array_equal(orc.field(f), dumps[3][f], err_msg=f)
    orc.close()


def test_build_recipe_patches_exactly_once():
    """Every textual patch of the reference build recipe matches exactly one site."""
    import build_ref
    src_path = os.path.join(build_ref.default_ref(), "les_combustion_solver.c")
    if not os.path.exists(src_path):
        pytest.skip("reference source not present")
    with open(src_path, encoding="utf-8") as f:
        src = f.read()
    patched = build_ref.patch_source(src, build_ref.CONFIGS["tiny"])
    assert "#define NX 24" in patched and "les_ref_after_step(t_loop, DT_sim)" in patched
    assert "#pragma omp parallel for if(!les_ref_serial_bc)" in patched
