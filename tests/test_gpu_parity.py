"""GPU parity: the CUDA solver step through the C ABI against the oracle and against the
reference's own outputs (tests/golden).

Tolerances (plain FP64 form), relative L2 per state field ||gpu - ref|| / ||ref||:
  * RHS intermediates of one calculate_RHS evaluation: 1e-12
  * whole state after 1 step: 1e-10; after 10 steps: 1e-8 (the parity tolerances the drop-in is held to)
  * dt: identical (it is a max-reduction of identical fields and a host formula)
  * SEM inflow face: bit-identical (the plane is summed in the reference's order)
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
TOL_RHS = 1e-12
TOL_1 = 1e-10
TOL_10 = 1e-8


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def worst(gpu_state, ref_state, fields=STATE):
    errs = {f: rel(gpu_state[f], ref_state[f]) for f in fields}
    k = max(errs, key=errs.get)
    return errs[k], k


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


@pytest.mark.parametrize("name,before,t_loop", [("tiny", 0, 0), ("small", 15, 0), ("small", 15, 500), ("c1", 8, 499)])
def test_rhs_intermediates(N, oracle_mod, name, before, t_loop):
    """One calculate_RHS (filter, mixture properties, nu_t, S_T, all k-arrays) on the same
    state, including the t_loop >= 500 WENO-gradient branch."""
    from lesgpu.config import preset
    cfg = preset(name)
    orc = oracle_mod.Oracle(cfg.as_dict())
    orc.step(before)
    ctx = N.Context(cfg)
    ctx.upload_attribute(orc.attribute())
    ctx.upload_state(orc.state())
    ctx.eval_rhs(t_loop)
    orc.rhs_only(t_loop)
    bad = []
    for k in N._INSPECT:
        r = rel(ctx.field(k), orc.field(k))
        if r > TOL_RHS:
            bad.append((k, r))
    for k in ["nu_t", "S_mag"]:
        r = rel(ctx.field(k), orc.field(k))
        if r > TOL_RHS:
            bad.append((k, r))
    ctx.close()
    orc.close()
    assert not bad, bad


def _run_gpu(N, cfg, steps, start=0, keep=()):
    sol = N.Solver(cfg, start_step=start)
    out, dts = {}, []
    for n in range(1, steps + 1):
        sol.step()
        dts.append(sol.last_dt)
        if n in keep:
            st = sol.state()
            st["nu_t"] = sol.field("nu_t")
            st["S_mag"] = sol.field("S_mag")
            out[n] = st
    sol.close()
    return out, dts


@pytest.mark.parametrize("case", ["tiny_s10", "tiny_w495", "small_s12"])
def test_steps_match_reference_fixtures(N, case):
    """Whole time steps against states written by the compiled reference."""
    from lesgpu.config import preset
    g = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    cfg = preset(str(g["config"]), seed=int(g["seed"]))
    keep = [int(x) for x in g["steps"]]
    out, dts = _run_gpu(N, cfg, len(g["dt"]), start=int(g["start"]), keep=keep)
    assert dts == list(g["dt"]), "dt sequence differs"
    for n in keep:
        ref = {f: g[f"s{n}_{f}"] for f in STATE + ["nu_t", "S_mag"]}
        e, f = worst(out[n], ref, STATE + ["nu_t", "S_mag"])
        tol = TOL_1 if n == 1 else TOL_10
        assert e <= tol, f"{case} step {n}: {f} rel L2 {e:.3e} > {tol}"


def test_ten_steps_64x32x32(N, oracle_mod):
    """The 64x32x32 / 200-eddy case, 10 steps against the oracle."""
    from lesgpu.config import preset
    cfg = preset("c1")
    orc = oracle_mod.Oracle(cfg.as_dict())
    sol = N.Solver(cfg)
    for n in range(1, 11):
        orc.step()
        sol.step()
        assert sol.last_dt == orc.dt, f"dt differs at step {n}"
        if n in (1, 10):
            e, f = worst(sol.state(), orc.state())
            assert e <= (TOL_1 if n == 1 else TOL_10), f"step {n}: {f} {e:.3e}"
    sol.close()
    orc.close()


def test_sem_inflow_face_bit_identical(N, oracle_mod):
    from lesgpu.config import preset
    cfg = preset("c1", seed=2024)
    orc = oracle_mod.Oracle(cfg.as_dict())
    sol = N.Solver(cfg)
    for _ in range(3):
        orc.step()
        sol.step()
        attr = orc.attribute()
        st = sol.state()
        inlet = attr[0] == 1
        for f in ("u", "v", "w"):
            np.testing.assert_array_equal(st[f][0][inlet], orc.field(f)[0][inlet])
    np.testing.assert_array_equal(sol.vortices(), orc.vortices())
    sol.close()
    orc.close()


def test_probe_lines_and_monitor(N, oracle_mod):
    from lesgpu.config import preset
    cfg = preset("small")
    sol = N.Solver(cfg)
    sol.step(3)
    st = sol.state()
    nut, smag = sol.field("nu_t"), sol.field("S_mag")
    stations = [2, 5, 9, 20]
    k = cfg.nz // 2
    lines = sol.ctx.probe_lines(stations, k)
    for q, i in enumerate(stations):
        want = np.stack([st["u"][i, :, k], st["v"][i, :, k], st["w"][i, :, k], st["G"][i, :, k],
                         nut[i, :, k], smag[i, :, k]], axis=1)
        np.testing.assert_array_equal(lines[q], want)
    mon = sol.ctx.monitor()
    dx, dy, dz = cfg.lx / cfg.nx, cfg.ly / cfg.ny, cfg.lz / cfg.nz
    mass = np.cumsum(((st["rho"].ravel() * dx) * dy) * dz)[-1]
    assert abs(mon[0] - mass) <= 1e-13 * mass
    assert mon[1] == st["T"].min() and mon[2] == st["T"].max()
    assert mon[3] == st["G"].min() and mon[4] == st["G"].max() and mon[5] == st["Y0"].min()
    sol.close()


def test_probe_and_monitor_files(N, oracle_mod, tmp_path):
    """Probe rows use the reference's G = 0.5 search and CSV format (les_combustion_solver.c:3403-3471)."""
    from lesgpu.config import preset
    cfg = preset("small")
    sol = N.Solver(cfg)
    # a state with a lateral flame edge on the probe line: burnt for j < 6
    st = sol.state()
    attr = sol.attribute()
    fluid = attr == 3
    G = st["G"].copy()
    G[:, :, :] = 0.0
    G[:, :6, :] = 1.0
    G[~fluid & (attr != 5)] = st["G"][~fluid & (attr != 5)]
    st["G"] = G
    sol.ctx.upload_state(st)
    sol.set_outputs(str(tmp_path), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    sol.step(1)
    rows = (tmp_path / "probe_data_flame_region_loc0.csv").read_text().splitlines()
    assert rows[0] == "timestep,x_location,y_flame,y_physical,y_relative,u,v,w,G,nu_t,S_mag"
    assert len(rows) == 1 + cfg.ny
    first = rows[1].split(",")
    assert first[0] == "0" and first[1] == "0.010"
    mon = (tmp_path / "simulation_monitor.csv").read_text().splitlines()
    assert mon[0].startswith("step,dt,total_mass") and mon[1].startswith("0,")
    sol.close()


def test_checkpoint_round_trip(N, tmp_path):
    from lesgpu.config import preset
    cfg = preset("tiny")
    a = N.Solver(cfg)
    a.step(4)
    path = str(tmp_path / "checkpoint.bin")
    a.save_checkpoint(path, 4)
    n = cfg.cells
    assert os.path.getsize(path) == 4 + 11 * 8 * n
    raw = np.fromfile(path, dtype=np.uint8)
    assert int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0]) == 4
    u = np.frombuffer(raw[4:4 + 8 * n].tobytes(), dtype=np.float64).reshape(cfg.nx, cfg.ny, cfg.nz)
    st = a.state()
    np.testing.assert_array_equal(u, st["u"])
    assert (tmp_path / "restart_info.txt").read_text() == "BINARY\n4\n"
    b = N.Solver(cfg)
    assert b.load_checkpoint(path) == 4
    for f in STATE:
        np.testing.assert_array_equal(b.state()[f], st[f])
    a.close()
    b.close()


def test_checkpoint_rejects_corrupt_file(N, tmp_path):
    from lesgpu.config import preset
    cfg = preset("tiny")
    s = N.Solver(cfg)
    bad = tmp_path / "short.bin"
    bad.write_bytes(b"\x00" * 100)
    with pytest.raises(N.LesgpuError) as e:
        s.load_checkpoint(str(bad))
    assert e.value.code == -4
    s.close()


def test_nonfinite_state_detected(N):
    from lesgpu.config import preset
    cfg = preset("tiny")
    s = N.Solver(cfg)
    assert s.ctx.check_finite("u")
    st = s.state()
    st["u"][5, 5, 5] = np.nan
    s.ctx.upload_state(st)
    assert not s.ctx.check_finite("u")
    s.close()


def test_call_order_errors(N):
    from lesgpu.config import preset
    cfg = preset("tiny")
    attr, st = N.initial_state(cfg)
    ctx = N.Context(cfg)
    with pytest.raises(N.LesgpuError) as e:
        ctx.step(1e-4, 0)
    assert e.value.code == -5
    ctx.upload_attribute(attr)
    ctx.upload_state(st)
    with pytest.raises(N.LesgpuError) as e:
        ctx.step(1e-4, 0)          # no inflow set for this step
    assert e.value.code == -5
    ctx.set_inflow(np.zeros((cfg.num_vortices, 7)), np.zeros((3, cfg.ny, cfg.nz)))
    with pytest.raises(N.LesgpuError) as e:
        ctx.step(-1.0, 0)
    assert e.value.code == -1
    ctx.close()


def test_fp32_precision_form_tracks_fp64(N):
    """The FP32-bulk form stays close to FP64 over a short run (full statistics parity is a
    long-run property checked by the profile comparison)."""
    from lesgpu.config import preset
    cfg = preset("c1")
    a = N.Solver(cfg, precision=N.FP64)
    b = N.Solver(cfg, precision=N.FP32)
    a.step(10)
    b.step(10)
    sa, sb = a.state(), b.state()
    for f in ("u", "T", "G", "rho"):
        assert np.isfinite(sb[f]).all()
        assert rel(sb[f], sa[f]) < 1e-3, f
    a.close()
    b.close()


def test_constant_division_matches_ieee(N):
    """The kernels evaluate divisions by constants as a reciprocal product with one fma
    correction; it must give the same bits as IEEE division for the divisors they use."""
    from lesgpu.config import preset
    from lesgpu import props
    divs = [6.0, 56.0, 1.6, 1.0, 0.03]
    for name in ("c1", "c2", "c3", "tiny"):
        c = preset(name)
        for d in (c.lx / c.nx, c.ly / c.ny, c.lz / c.nz):
            divs += [d, 2.0 * d, d * d]
        divs.append(2.0 * c.accel_width * c.accel_width)
    divs += [m / 1000.0 for m in props.synthetic_species().mw]
    # the TENO weight sums w0 + w1 + w2 of every cut-off pattern (kernel operation order)
    for q in range(1, 8):
        divs.append((q & 1) * 0.1 + ((q >> 1) & 1) * 0.6 + ((q >> 2) & 1) * 0.3)
    assert N.selfcheck_division(divs, 1 << 21) == 0


def test_shared_denominator_division_matches_ieee(N):
    """Quotients sharing a denominator are computed from one reciprocal y = 1/b (IEEE) and a
    corrected product; the same check with random divisors over the exponent range the
    properties use (and significands near 1 and 2) must find no difference from IEEE."""
    rng = np.random.default_rng(5)
    sig = rng.uniform(1.0, 2.0, 2048)
    sig[:128] = 2.0 - rng.integers(1, 1 << 20, 128) * 2.0 ** -52
    sig[128:256] = 1.0 + rng.integers(1, 1 << 20, 128) * 2.0 ** -52
    d = np.ldexp(sig, rng.integers(-40, 40, 2048)) * np.where(rng.random(2048) < 0.5, 1.0, -1.0)
    assert N.selfcheck_division(d, 1 << 17, seed=99) == 0


def test_device_loop_matches_host_loop(N, tmp_path):
    """The device-resident loop (dt, vortex recycling and inflow noise on the GPU through the
    rand() jump-ahead, graph-replayed steps) is bit-identical to the host-driven loop,
    including the rand() stream handed back afterwards and the probe/monitor files."""
    from lesgpu.config import preset
    cfg = preset("c1", seed=4242)
    a, b = N.Solver(cfg), N.Solver(cfg)
    da, db = tmp_path / "host", tmp_path / "dev"
    da.mkdir()
    db.mkdir()
    a.set_outputs(str(da), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    b.set_outputs(str(db), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
    a.step(23)
    b.run_device(23, chunk=7)
    assert a.t_loop == b.t_loop == 23
    assert a.last_dt == b.last_dt
    np.testing.assert_array_equal(a.vortices(), b.vortices())
    sa, sb = a.state(), b.state()
    for f in STATE:
        np.testing.assert_array_equal(sa[f], sb[f], err_msg=f)
    # host-driven steps continue from the handed-back rand() window
    a.step(2)
    b.step(2)
    np.testing.assert_array_equal(a.vortices(), b.vortices())
    np.testing.assert_array_equal(a.state()["u"], b.state()["u"])
    for fn in ["simulation_monitor.csv"] + [f"probe_data_flame_region_loc{n}.csv" for n in range(7)]:
        assert (da / fn).read_text() == (db / fn).read_text(), fn
    a.close()
    b.close()


def test_device_loop_chunking_invariant(N, tmp_path):
    """Splitting a device-loop run into chunks (history slots, graph replays across chunk
    boundaries, checkpoint stops at t % 50 == 0) does not change the result or the files."""
    from lesgpu.config import preset
    cfg = preset("small")
    outs = []
    for chunk in (3, 64):
        d = tmp_path / f"c{chunk}"
        d.mkdir()
        s = N.Solver(cfg)
        s.set_outputs(str(d), N.LES_OUT_PROBES | N.LES_OUT_MONITOR | N.LES_OUT_CHECKPOINT)
        s.run_device(53, chunk=chunk)
        outs.append((s.state(), s.vortices(), s.last_dt, d))
        s.close()
    (sa, va, ta, da), (sb, vb, tb, db) = outs
    assert ta == tb
    np.testing.assert_array_equal(va, vb)
    for f in STATE:
        np.testing.assert_array_equal(sa[f], sb[f], err_msg=f)
    for fn in ["simulation_monitor.csv", "checkpoint.bin", "restart_info.txt"]:
        assert (da / fn).read_bytes() == (db / fn).read_bytes(), fn
    assert (da / "restart_info.txt").read_text() == "BINARY\n50\n"
