"""Ensembles, group graphs and tile selection on the GPU.

* members advanced together by one multi-stream graph per step give bit-identical states
  and output files to the same members run alone with the same tiles;
* the thread-block tile changes results only through the summation order of <rho_f>
  (relative L2 difference at rounding level, 1e-13 after three steps);
* lesgpu_autotune leaves the state, the dt inputs and the counters as they were.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
TOL_TILE = 1e-13


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _files(d):
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))}


def test_ensemble_members_match_solo_runs(N, tmp_path):
    from lesgpu.config import preset
    from lesgpu.ensemble import Ensemble
    cfgs = [preset("tiny", seed=11, cs_unburned=0.09, relax=2500.0),
            preset("small", seed=12, accel_strength=3.5),
            preset("c1", seed=13, cs_unburned=0.2, relax=100.0)]
    ens = Ensemble(cfgs, precision=N.FP64, autotune=True)
    dirs = []
    for q, m in enumerate(ens.members):
        d = tmp_path / f"ens{q}"
        d.mkdir()
        m.set_outputs(str(d), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
        dirs.append(str(d))
    ens.run(12, chunk=5)
    got = [m.state() for m in ens.members]
    tiles = [m.ctx.get_tiles() for m in ens.members]
    t_loops = [m.t_loop for m in ens.members]
    ens.close()
    for q, (cfg, st, tl) in enumerate(zip(cfgs, got, tiles)):
        assert all(0 <= t < len(N.Context.TILES) for t in tl)
        solo = N.Solver(cfg)
        solo.ctx.set_tiles(tl)
        d = tmp_path / f"solo{q}"
        d.mkdir()
        solo.set_outputs(str(d), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
        solo.run_device(12, chunk=12)
        ref = solo.state()
        assert t_loops[q] == solo.t_loop == 12
        for f in STATE:
            np.testing.assert_array_equal(st[f], ref[f], err_msg=f"member {q}: {f}")
        assert _files(dirs[q]) == _files(str(d)), f"member {q}: output files differ"
        solo.close()


def test_ensemble_continues_across_runs(N):
    """Two ensemble runs in a row equal one run of the summed length."""
    from lesgpu.config import preset
    from lesgpu.ensemble import Ensemble
    cfgs = [preset("tiny", seed=3), preset("small", seed=4)]
    a = Ensemble(cfgs, precision=N.FP64, autotune=False)
    a.run(4, chunk=4)
    a.run(5, chunk=3)
    sa = [m.state() for m in a.members]
    a.close()
    b = Ensemble(cfgs, precision=N.FP64, autotune=False)
    b.run(9, chunk=9)
    sb = [m.state() for m in b.members]
    b.close()
    for x, y in zip(sa, sb):
        for f in STATE:
            np.testing.assert_array_equal(x[f], y[f])


def _class_tiles(N, t):
    # a 512-thread tile (index 8 on) serves the strain, flow and scalar classes; the filter
    # and EOS classes keep tile 0 then
    bx, by, bz = N.Context.TILES[t]
    wide = bx * by * bz > 256
    return [0 if (wide and c in (0, 4)) else t for c in range(5)]


def test_tiles_change_only_rounding(N):
    from lesgpu.config import preset
    cfg = preset("small")
    ref = None
    for t in range(len(N.Context.TILES)):
        s = N.Solver(cfg)
        tl = _class_tiles(N, t)
        s.ctx.set_tiles(tl)
        assert s.ctx.get_tiles() == tl
        s.step(3)
        st = s.state()
        s.close()
        if ref is None:
            ref = st
            continue
        for f in STATE:
            if tl[0] == 0:
                # same filter tile: the <rho_f> partials are summed in the same order, and the
                # strain, flow and scalar passes reduce nothing, so the bits are the same
                np.testing.assert_array_equal(st[f], ref[f], err_msg=f"{t} {f}")
            else:
                assert rel(st[f], ref[f]) < TOL_TILE, (t, f, rel(st[f], ref[f]))


def test_wide_tiles_refused_for_reducing_classes(N):
    from lesgpu.config import preset
    s = N.Solver(preset("tiny"))
    before = s.ctx.get_tiles()
    for bad in ([8, 0, 0, 0, 0], [0, 0, 0, 0, 12], [0, 13, 0, 0, 0], [0, 0, 0, -1, 0]):
        with pytest.raises(N.LesgpuError):
            s.ctx.set_tiles(bad)
        assert s.ctx.get_tiles() == before
    s.ctx.set_tiles([7, 8, 10, 12, 7])
    assert s.ctx.get_tiles() == [7, 8, 10, 12, 7]
    s.close()


def test_autotune_leaves_state_and_dt_inputs(N):
    from lesgpu.config import preset
    cfg = preset("small", seed=5)
    a = N.Solver(cfg)
    a.step(2)
    before = a.ctx.dt_inputs()
    tiles, ms = a.ctx.autotune(reps=2)
    nt = len(N.Context.TILES)
    assert len(tiles) == 5 and all(0 <= t < nt for t in tiles)
    assert ms.shape == (4, nt) and np.all(ms > 0) and np.all(np.isfinite(ms))
    assert tiles[4] == tiles[0]
    for c in range(4):
        assert ms[c, tiles[c]] == ms[c].min()
    assert a.ctx.dt_inputs() == before
    a.step(3)
    b = N.Solver(cfg)
    b.step(2)
    b.ctx.set_tiles(tiles)
    b.step(3)
    sa, sb = a.state(), b.state()
    for f in STATE:
        np.testing.assert_array_equal(sa[f], sb[f], err_msg=f)
    assert a.t_loop == b.t_loop == 5
    a.close()
    b.close()


def test_group_requires_loop_sessions(N):
    from lesgpu.config import preset
    L = N.lib()
    s = N.Solver(preset("tiny"))
    arr = (C.c_void_p * 1)(s.ctx._h.value)
    g = C.c_void_p()
    assert L.lesgpu_group_create(arr, 1, C.byref(g)) == N.LESGPU_ESTATE
    s.loop_begin(chunk=4)
    assert L.lesgpu_group_create(arr, 1, C.byref(g)) == 0
    assert L.lesgpu_group_run(g, 5) == N.LESGPU_EINVAL      # beyond the history capacity
    assert L.lesgpu_group_run(g, 2) == 0
    L.lesgpu_group_destroy(g)
    s.loop_end()
    assert s.t_loop == 0        # steps queued through the raw group are not collected
    dup = (C.c_void_p * 2)(s.ctx._h.value, s.ctx._h.value)
    s.loop_begin(chunk=4)
    assert L.lesgpu_group_create(dup, 2, C.byref(g)) == N.LESGPU_EINVAL
    s.loop_end()
    s.close()


def test_optimisation_campaign_on_ensembles(N, tmp_path):
    """Two rounds of three proposals, each round one ensemble; every trial is scored from its
    own probe file and registered."""
    from lesgpu.config import preset
    from lesgpu.optimizer import run_campaign
    opt = run_campaign(preset("small", seed=4), rounds=2, batch=3, steps=25, precision=N.FP32,
                       workdir=str(tmp_path), seed=1, log=lambda *_: None)
    assert len(opt.y_obs) == 6
    assert all(np.isfinite(opt.y_obs))
    assert os.path.exists(tmp_path / "optimization_history.json")
    trials = sorted(p for p in os.listdir(tmp_path) if p.startswith("round"))
    assert len(trials) == 6
    for t in trials:
        assert os.path.exists(tmp_path / t / "probe_data_flame_region_loc0.csv")


@pytest.mark.parametrize("name,prec", [("c1", "fp64"), ("small", "fp64"), ("c1", "fp32"), ("e96", "fp64")])
def test_staged_scalar_pass_gives_the_same_bits(N, name, prec):
    """The scalar pass reading its stencil fields from shared-memory planes filled by tensor
    copies runs the same arithmetic as the plain pass: in FP64 (no FMA contraction) identical
    states after the device loop and host-driven steps, and no copy timed out; in FP32 the
    two kernels may contract products into FMAs differently, so they agree to FP32 rounding."""
    from lesgpu.config import preset
    P = N.FP64 if prec == "fp64" else N.FP32
    cfg = preset(name, seed=17)
    out = []
    for staged in (False, True):
        s = N.Solver(cfg, precision=P)
        if staged:
            s.ctx.set_scalar_staging(True)
            assert s.ctx.get_scalar_staging()
        s.run_device(9, chunk=4)
        s.step(2)
        out.append(s.state())
        s.close()
    for f in STATE:
        if prec == "fp64":
            np.testing.assert_array_equal(out[0][f], out[1][f], err_msg=f)
        else:
            np.testing.assert_allclose(out[1][f], out[0][f], rtol=1e-5, atol=1e-9, err_msg=f)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batched_ensemble_matches_solo_runs(N, prec, tmp_path):
    """The batched form (one launch per RK pass over the members of a grid shape, each block
    reading its member's arena, reductions and model constants from the member table) against
    solo runs with the same tiles: FP64 members bit-identical, output files included; FP32
    members within 1e-6 relative L2 per field (the FP32 unit is built with FMA contraction,
    and the batched instantiation of a kernel may contract differently from the solo one).
    Two grid shapes, members with different model constants and seeds, and one member whose
    other constants differ (its own batch)."""
    from lesgpu.config import preset
    from lesgpu.ensemble import Ensemble
    P = N.FP64 if prec == "fp64" else N.FP32
    cfgs = [preset("tiny", seed=21, cs_unburned=0.09, relax=2500.0),
            preset("small", seed=22, accel_strength=3.5, cs_burnt=0.3),
            preset("tiny", seed=23, cs_unburned=0.2, accel_center=0.5, accel_width=0.2, cs_flame_boost=0.1),
            preset("small", seed=24, relax=100.0),
            preset("tiny", seed=25, s_l=0.45, courant=0.2)]
    ens = Ensemble(cfgs, precision=P, autotune=True, batched=True, per_batch=0 if prec == "fp64" else 2)
    dirs = []
    for q, m in enumerate(ens.members):
        d = tmp_path / f"ens{q}"
        d.mkdir()
        m.set_outputs(str(d), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
        dirs.append(str(d))
    ens.run(9, chunk=4)
    ens.run(5, chunk=5)
    got = [m.state() for m in ens.members]
    tiles = [m.ctx.get_tiles() for m in ens.members]
    ens.close()
    for q, (cfg, st, tl) in enumerate(zip(cfgs, got, tiles)):
        solo = N.Solver(cfg, precision=P)
        solo.ctx.set_tiles(tl)
        d = tmp_path / f"solo{q}"
        d.mkdir()
        solo.set_outputs(str(d), N.LES_OUT_PROBES | N.LES_OUT_MONITOR)
        solo.run_device(14, chunk=14)
        ref = solo.state()
        if P == N.FP64:
            for f in STATE:
                np.testing.assert_array_equal(st[f], ref[f], err_msg=f"member {q}: {f}")
            assert _files(dirs[q]) == _files(str(d)), f"member {q}: output files differ"
        else:
            for f in STATE:
                e = np.linalg.norm(st[f] - ref[f]) / max(np.linalg.norm(ref[f]), 1e-300)
                assert e <= 1e-6, f"member {q}: {f} rel L2 {e:.2e}"
        solo.close()


def test_batched_group_forms_batches_by_shape_and_constants(N):
    """Members batch together only when grid, precision, tiles and every kernel constant but
    the optimiser's agree (the Courant number only enters each member's own dt)."""
    import ctypes as C
    from lesgpu.config import preset
    cfgs = [preset("tiny", seed=1), preset("tiny", seed=2, cs_unburned=0.1, relax=10.0), preset("small", seed=3),
            preset("tiny", seed=4, s_l=0.45), preset("small", seed=5, accel_strength=1.0, courant=0.2)]
    sols = [N.Solver(c) for c in cfgs]
    for s in sols:
        s.loop_begin(chunk=4)
    arr = (C.c_void_p * len(sols))(*[s.ctx._h.value for s in sols])
    g = C.c_void_p()
    assert N.lib().lesgpu_group_create_batched(arr, len(sols), 0, C.byref(g)) == 0
    assert N.lib().lesgpu_group_batches(g) == 3          # {tiny 1, 2}, {small 3, 5}, {tiny 4}
    assert N.lib().lesgpu_group_run(g, 3) == 0
    N.lib().lesgpu_group_destroy(g)
    g = C.c_void_p()
    assert N.lib().lesgpu_group_create_batched(arr, len(sols), 1, C.byref(g)) == 0
    assert N.lib().lesgpu_group_batches(g) == 5          # at most one member per batch
    N.lib().lesgpu_group_destroy(g)
    for s in sols:
        s.loop_end()
        s.close()
