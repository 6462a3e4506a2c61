"""The drop-in run inside the reference's own main(): the reference solver with the first C
block of INTEGRATION.md spliced into it (gpu_begin / gpu_step replacing the loop body
les_combustion_solver.c:4399-4555), built by tests/dropin/build_dropin.py against
liblesgpu.so, runs 50 steps of the 64x32x32 / 200-eddy case beside the unmodified reference.

Both are the same C program apart from those lines: same initialisation, same host rand()
stream (the drop-in draws the vortex recycling and the inflow noise on the host, in the
reference's order), same probe / monitor / checkpoint writers.  Compared: the state after
50 steps (relative L2 1e-8 per field, the 10-step parity bar), the dt sequence (1e-13
relative), the final checkpoint.bin both programs write at exit, the probe files and the
monitor file (one unit of the last printed digit).
"""
import os

import numpy as np
import pytest

from refcompare import compare_monitor, compare_probes, rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "tests", "dropin", "_build", "c1", "les_dropin")
STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]


def _checkpoint(path, shape):
    raw = np.fromfile(path, dtype=np.uint8)
    n = shape[0] * shape[1] * shape[2]
    assert raw.size == 4 + 11 * 8 * n
    arr = np.frombuffer(raw[4:].tobytes(), dtype=np.float64).reshape(11, *shape)
    return int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0]), {f: arr[q] for q, f in enumerate(STATE)}


def test_dropin_inside_reference_main_matches_reference(lesgpu_native, cuda_device, oracle_mod, tmp_path):
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in harness not built (tests/dropin/build_dropin.py needs the reference source)")
    if not oracle_mod.ref_available("c1"):
        pytest.skip("compiled reference for c1 not present")
    steps = 50
    threads = os.cpu_count() or 1
    env = {"LES_REF_SERIAL_BC": 1}
    ref_dir, gpu_dir = str(tmp_path / "ref"), str(tmp_path / "dropin")
    ref, ref_meta = oracle_mod.run_reference("c1", steps, seed=1234, dump_every=steps, threads=threads,
                                             env_extra=env, keep_dir=ref_dir)
    gpu, gpu_meta = oracle_mod.run_reference("c1", steps, seed=1234, dump_every=steps, threads=threads,
                                             env_extra=env, keep_dir=gpu_dir, binary=DROPIN)
    dt_r = np.array([t[1] for t in ref_meta["times"]])
    dt_g = np.array([t[1] for t in gpu_meta["times"]])
    assert len(dt_g) == len(dt_r) == steps
    dt_err = float(np.max(np.abs(dt_g - dt_r) / dt_r))
    errs = {f: rel(gpu[steps][f], ref[steps][f]) for f in STATE + ["nu_t", "S_mag"]}
    k = max(errs, key=errs.get)
    print(f"\n[drop-in c1 x {steps}] dt max rel diff {dt_err:.2e}; state worst rel L2 {errs[k]:.2e} ({k})")
    assert dt_err <= 1e-13
    assert errs[k] <= 1e-8, errs
    shape = ref[steps]["u"].shape
    tr, cr = _checkpoint(os.path.join(ref_dir, "checkpoint.bin"), shape)
    tg, cg = _checkpoint(os.path.join(gpu_dir, "checkpoint.bin"), shape)
    assert tr == tg
    ck = {f: rel(cg[f], cr[f]) for f in STATE}
    assert max(ck.values()) <= 1e-8, ck
    with open(os.path.join(ref_dir, "restart_info.txt")) as f1, open(os.path.join(gpu_dir, "restart_info.txt")) as f2:
        assert f1.read() == f2.read()
    pw = compare_probes(gpu_meta["probes"], ref_meta["probes"])
    compare_monitor(gpu_meta["monitor"], ref_meta["monitor"])
    print(f"[drop-in c1 x {steps}] checkpoint.bin worst rel L2 {max(ck.values()):.2e}; probe rows max |diff| {pw:.1e}")
