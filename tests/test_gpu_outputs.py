"""Outputs of the time loop beyond the state, on the GPU:

* time averages (update_time_averages, les_combustion_solver.c:3166-3191): the device sums
  equal the sums of the oracle's per-step states (rel. 1e-12; the states themselves agree to
  ~1e-14), host-driven and device loop give the same bits, stats_backup.bin round-trips, and
  the Reynolds stresses follow calculate_resolved_reynolds_stresses (:3194-3217);
* the point time series (:4557-4568, flush_point_data :3824-3850): one file per measurement
  point, the same from host-driven and device-loop runs, values equal to the oracle's state
  at the point to the file's 6 decimals.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_AVG = 1e-12


@pytest.fixture(scope="module")
def N(lesgpu_native, cuda_device):
    return lesgpu_native


def _oracle_sums(oracle_mod, cfg, steps, start):
    orc = oracle_mod.Oracle(cfg.as_dict())
    sums = None
    n = 0
    for t in range(steps):
        orc.step()
        if t < start:
            continue
        u, v, w, G = (orc.field(k) for k in ("u", "v", "w", "G"))
        add = {"u": u, "v": v, "w": w, "G": G, "uu": u * u, "vv": v * v, "ww": w * w, "uv": u * v,
               "uw": u * w, "vw": v * w}
        if sums is None:
            sums = {k: np.zeros_like(u) for k in add}
        for k in add:
            sums[k] = sums[k] + add[k]
        n += 1
    orc.close()
    return sums, n


def test_time_averages_match_oracle(N, oracle_mod):
    from lesgpu.config import preset
    cfg = preset("tiny", seed=21)
    steps, start = 14, 5
    ref, nref = _oracle_sums(oracle_mod, cfg, steps, start)
    host = N.Solver(cfg)
    host.set_averaging(start)
    host.step(steps)
    hs, hn = host.average_sums()
    dev = N.Solver(cfg)
    dev.set_averaging(start)
    dev.run_device(steps, chunk=4)
    ds, dn = dev.average_sums()
    assert hn == dn == nref == steps - start
    for k in N.AVG_NAMES:
        np.testing.assert_array_equal(hs[k], ds[k], err_msg=k)
        nb = np.linalg.norm(ref[k])
        assert np.linalg.norm(hs[k] - ref[k]) / (nb if nb > 0 else 1.0) < TOL_AVG, k
    st, n = host.reynolds_stresses()
    assert n == nref
    au = hs["u"] / n
    av = hs["v"] / n
    np.testing.assert_array_equal(st["uu"], hs["uu"] / n - au * au)
    np.testing.assert_array_equal(st["uv"], hs["uv"] / n - au * av)
    np.testing.assert_array_equal(st["G_mean"], hs["G"] / n)
    host.close()
    dev.close()


def test_stats_backup_round_trip(N, tmp_path):
    from lesgpu.config import preset
    cfg = preset("tiny", seed=3)
    a = N.Solver(cfg)
    a.set_averaging(0)
    a.step(6)
    path = str(tmp_path / "stats_backup.bin")
    a.save_stats(path)
    sa, na = a.average_sums()
    raw = np.fromfile(path, dtype=np.uint8)
    assert raw.size == 4 + 10 * 8 * cfg.cells
    assert int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0]) == na == 6
    b = N.Solver(cfg)
    b.set_averaging(0)
    b.load_stats(path)
    sb, nb = b.average_sums()
    assert nb == na
    for k in N.AVG_NAMES:
        np.testing.assert_array_equal(sa[k], sb[k])
    # the file layout: u, v, w, uu, vv, ww, uv, uw, vw, G after the count
    body = np.frombuffer(raw[4:].tobytes(), dtype=np.float64).reshape(10, -1)
    for q, k in enumerate(N.AVG_NAMES):
        np.testing.assert_array_equal(body[q], sa[k].ravel())
    # checkpoint steps write it next to checkpoint.bin
    c = N.Solver(cfg)
    c.set_averaging(0)
    os.makedirs(tmp_path / "run")
    c.set_outputs(str(tmp_path / "run"), N.LES_OUT_CHECKPOINT)
    c.run_device(51, chunk=64)
    assert os.path.exists(tmp_path / "run" / "stats_backup.bin")
    assert os.path.exists(tmp_path / "run" / "checkpoint.bin")
    with pytest.raises(N.LesgpuError):
        c.load_stats(str(tmp_path / "missing.bin"))
    for s in (a, b, c):
        s.close()


def _point_files(d):
    return {f: open(os.path.join(d, f)).read() for f in sorted(os.listdir(d)) if f.startswith("LES_point_data")}


def test_point_time_series(N, oracle_mod, tmp_path):
    from lesgpu.config import preset
    cfg = preset("small", seed=8)
    steps = 57
    dh, dd = tmp_path / "host", tmp_path / "dev"
    dh.mkdir()
    dd.mkdir()
    h = N.Solver(cfg)
    h.set_outputs(str(dh), N.LES_OUT_POINTS)
    h.step(steps)
    h.flush()
    d = N.Solver(cfg)
    d.set_outputs(str(dd), N.LES_OUT_POINTS)
    d.run_device(steps, chunk=16)
    d.close()                                  # destroying flushes the rest
    fh, fd = _point_files(str(dh)), _point_files(str(dd))
    assert fh == fd and len(fh) > 0
    # the points: 4D and 8D downstream, axis and shear layer, k = NZ/2
    dx, dy = cfg.lx / cfg.nx, cfg.ly / cfg.ny
    i4, i8 = int(4.0 * cfg.inlet_radius / dx), int(8.0 * cfg.inlet_radius / dx)
    js = int(cfg.inlet_radius / dy)
    want = {(i, j) for i in (i4, i8) if i < cfg.nx for j in (0, js)}
    got = {(int(f.split("_i")[1].split("_")[0]), int(f.split("_j")[1].split("_")[0])) for f in fh}
    assert got == want
    orc = oracle_mod.Oracle(cfg.as_dict())
    rows = {f: np.loadtxt(os.path.join(str(dh), f), delimiter=",", skiprows=1, ndmin=2) for f in fh}
    for f, r in rows.items():
        assert r.shape == (steps, 4)
    for t in range(steps):
        orc.step()
        for f, r in rows.items():
            i = int(f.split("_i")[1].split("_")[0])
            j = int(f.split("_j")[1].split("_")[0])
            k = int(f.split("_k")[1].split(".")[0])
            assert k == cfg.nz // 2
            ref = [orc.field(x)[i, j, k] for x in ("u", "v", "w", "G")]
            np.testing.assert_allclose(r[t], ref, atol=1.5e-6, rtol=0)
    orc.close()
    h.close()


def _golden_outputs():
    from conftest import GOLDEN
    return np.load(os.path.join(GOLDEN, "outputs_ref.npz"))


def _vtk_sections(text):
    """{name: values} of a legacy ASCII VTK file; 'points' for the coordinates."""
    lines = text.splitlines()
    out, q = {}, 0
    while q < len(lines):
        ln = lines[q]
        if ln.startswith("POINTS"):
            n = int(ln.split()[1])
            out["points"] = np.array([list(map(float, lines[q + 1 + r].split())) for r in range(n)])
            q += n + 1
        elif ln.startswith("VECTORS") or ln.startswith("SCALARS"):
            name = ln.split()[1]
            q += 1
            if lines[q].startswith("LOOKUP_TABLE"):
                q += 1
            vals = []
            while q < len(lines) and lines[q] and not lines[q][0].isalpha():
                vals.append(list(map(float, lines[q].split())))
                q += 1
            out[name] = np.array(vals)
        else:
            q += 1
    return out


def test_vtk_matches_reference_file(N, tmp_path):
    """output_vtk of the 24x12x16 case after 10 steps, against the reference's own file;
    values agree to the file's printed precision."""
    from lesgpu.config import preset
    z = _golden_outputs()
    ref_text = z["vtk_tiny_s10"].tobytes().decode()
    s = N.Solver(preset("tiny"))
    s.set_outputs(str(tmp_path), N.LES_OUT_VTK)
    s.step(10)
    s.flush()
    s.close()
    ours_text = open(tmp_path / "Premixed_C3H8_Air_0010.vtk").read()
    assert ours_text.splitlines()[:6] == ref_text.splitlines()[:6]
    a, b = _vtk_sections(ours_text), _vtk_sections(ref_text)
    assert list(a) == list(b)
    for k in b:
        assert a[k].shape == b[k].shape, k
        scale = np.maximum(np.abs(b[k]), 1e-30)
        err = np.abs(a[k] - b[k])
        # %.6f fields: 1e-6 absolute; %.6e fields: 1e-6 relative (plus one unit of rounding)
        ok = (err <= 1.5e-6) | (err <= 2e-6 * scale)
        assert ok.all(), (k, float(err.max()))
    assert np.abs(a["grad_G_magnitude"]).max() > 0


def test_point_files_match_reference(N, tmp_path):
    """The point time series of the 40x16x24 case (seed 77) over 60 steps -- flushed at step 50
    and at the end of the run -- against the reference's files."""
    from lesgpu.config import preset
    z = _golden_outputs()
    names = [str(x) for x in z["point_names"]]
    assert names
    s = N.Solver(preset("small", seed=77))
    s.set_outputs(str(tmp_path), N.LES_OUT_POINTS)
    s.run_device(60, chunk=32)
    s.flush()
    s.close()
    got = sorted(f for f in os.listdir(tmp_path) if f.startswith("LES_point_data"))
    assert got == names
    for q, f in enumerate(names):
        ref = z[f"point_{q}"].tobytes().decode().splitlines()
        ours = open(tmp_path / f).read().splitlines()
        assert ours[0] == ref[0] == "u,v,w,G"
        a = np.array([list(map(float, r.split(","))) for r in ours[1:]])
        b = np.array([list(map(float, r.split(","))) for r in ref[1:]])
        assert a.shape == b.shape == (60, 4)
        np.testing.assert_allclose(a, b, atol=1.5e-6, rtol=0)
