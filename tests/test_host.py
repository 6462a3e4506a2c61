"""Host-side logic of the C driver, checked on the CPU (no GPU calls).

The rand() stream, start-up state, SEM vortex bookkeeping, inflow noise and dt formula
must be bit-identical to the reference's (they feed the GPU step unchanged)."""
import ctypes
import os

import numpy as np
import pytest


def test_rng_matches_glibc_rand(lesgpu_native):
    libc = ctypes.CDLL("libc.so.6")
    for seed in [0, 1, 1234, 77, 2**31 - 1, 2**31, 2**32 - 1, 987654321]:
        libc.srand(ctypes.c_uint(seed))
        ref = [libc.rand() for _ in range(3000)]
        g = lesgpu_native.Rng(seed)
        assert [g.next() for _ in range(3000)] == ref, f"seed {seed}"


@pytest.mark.parametrize("name", ["tiny", "small", "c1"])
def test_initial_state_matches_oracle(lesgpu_native, oracle_mod, name):
    from lesgpu.config import preset
    cfg = preset(name)
    attr, st = lesgpu_native.initial_state(cfg)
    orc = oracle_mod.Oracle(cfg.as_dict())
    np.testing.assert_array_equal(attr, orc.attribute())
    for k, v in st.items():
        np.testing.assert_array_equal(v, orc.field(k), err_msg=k)
    orc.close()


def test_attribute_codes(lesgpu_native):
    """Attribute layout of setting() (les_combustion_solver.c:1151-1181)."""
    from lesgpu.config import preset
    cfg = preset("c1")
    attr, _ = lesgpu_native.initial_state(cfg)
    assert set(np.unique(attr)) == {1, 2, 3, 4, 5}
    assert (attr[-1] == 2).all()
    assert (attr[1:-1, 0, :] == 5).all()
    assert (attr[1:-1, -1, :] == 4).all() and (attr[1:-1, 1:-1, 0] == 4).all()
    assert (attr[1:-1, 1:-1, 1:-1] == 3).all()
    inlet = attr[0] == 1
    jj, kk = np.nonzero(inlet)
    dy, dz = cfg.ly / cfg.ny, cfg.lz / cfg.nz
    d2 = (jj * dy) ** 2 + (kk * dz - cfg.lz / 2) ** 2
    assert (d2 <= cfg.inlet_radius ** 2 + 1e-15).all()


def test_vortices_and_noise_track_oracle(lesgpu_native, oracle_mod):
    from lesgpu.config import preset
    N = lesgpu_native
    cfg = preset("small", seed=31337)
    c = N.LesgpuConfig.from_config(cfg)
    g = N.Rng(cfg.seed)
    vort = np.zeros((cfg.num_vortices, 7))
    N.lib().les_vortices_init(ctypes.byref(g._s), ctypes.byref(c), vort.ctypes.data)
    orc = oracle_mod.Oracle(cfg.as_dict())
    np.testing.assert_array_equal(vort, orc.vortices())
    attr = np.ascontiguousarray(orc.attribute()[0], dtype=np.int32)
    noise = np.zeros((3, cfg.ny, cfg.nz))
    for _ in range(6):
        orc.step()
        N.lib().les_vortices_update(ctypes.byref(g._s), ctypes.byref(c), vort.ctypes.data, orc.dt)
        N.lib().les_inflow_noise(ctypes.byref(g._s), attr.ctypes.data, cfg.ny, cfg.nz, noise.ctypes.data)
        np.testing.assert_array_equal(vort, orc.vortices())
    # after the noise draws the streams are aligned: the next draw is the same
    assert g.next() == ctypes.CDLL("libc.so.6").rand()
    orc.close()


def test_dt_formula(lesgpu_native, oracle_mod):
    from lesgpu.config import preset
    N = lesgpu_native
    cfg = preset("tiny")
    c = N.LesgpuConfig.from_config(cfg)
    # first step: nu = alpha = 0 (never initialised in the reference), |u|max = inlet velocity
    orc = oracle_mod.Oracle(cfg.as_dict())
    orc.step()
    assert N.lib().les_dt(ctypes.byref(c), 5.0, 0.0, 0.0) == orc.dt
    dx = cfg.lx / cfg.nx
    want = min(cfg.courant * dx / (7.0 + 1e-10), cfg.courant_diffusion * (dx * dx) / (2e-4 + 1e-10))
    assert N.lib().les_dt(ctypes.byref(c), 7.0, 2e-4, 1e-4) == want
    orc.close()


def test_species_loader_matches_reader(lesgpu_native):
    from lesgpu import props
    sp = lesgpu_native.load_species()
    r = props.read_species(lesgpu_native.CHEM_BIN, lesgpu_native.TRAN_BIN)
    assert list(sp.mw) == r.mw and list(sp.t_mid) == r.t_mid
    assert [list(x) for x in sp.nasa_low] == r.nasa_low and [list(x) for x in sp.nasa_high] == r.nasa_high
    assert [list(x) for x in sp.eta] == r.eta and [list(x) for x in sp.lam] == r.lam
    assert [[list(y) for y in x] for x in sp.dcoef] == r.dcoef


def test_species_files_are_the_synthetic_set():
    from lesgpu import props
    from lesgpu.native import CHEM_BIN, TRAN_BIN
    r = props.read_species(CHEM_BIN, TRAN_BIN)
    s = props.synthetic_species()
    assert r.mw == s.mw and r.dcoef == s.dcoef and r.nasa_high == s.nasa_high


def test_species_loader_rejects_bad_files(lesgpu_native, tmp_path):
    bad = tmp_path / "chem.bin"
    bad.write_bytes(b"\x10\x00\x00\x00short")
    with pytest.raises(lesgpu_native.LesgpuError) as e:
        lesgpu_native.load_species(str(bad), lesgpu_native.TRAN_BIN)
    assert e.value.code == -4
    with pytest.raises(lesgpu_native.LesgpuError):
        lesgpu_native.load_species(str(tmp_path / "missing.bin"), lesgpu_native.TRAN_BIN)


def test_presets_match_reference_build_configs():
    """The named grids agree with the macro values the reference oracle is compiled with."""
    import build_ref
    from lesgpu.config import preset
    for name, m in build_ref.CONFIGS.items():
        c = preset(name)
        assert (c.nx, c.ny, c.nz) == (m["nx"], m["ny"], m["nz"])
        assert (c.lx, c.ly, c.lz) == (m["lx"], m["ly"], m["lz"])
        assert c.num_vortices == m["nv"] and c.initial_flame_front_i == m["i_f"]
        assert c.inlet_velocity == m["u_in"] and c.turbulence_intensity == m["ti"]
        assert c.length_scale == m["ell"] and c.courant == m["courant"]


def test_ensemble_parameter_sets():
    """The batched-ensemble workload: 64 sets, CS_UNBURNED in [0.08, 0.22], strength in
    [0, 2] x default, nudging in [0, 1] x default, grids alternating, reproducible."""
    from lesgpu.ensemble import ensemble_configs
    a, b = ensemble_configs(64, seed=5), ensemble_configs(64, seed=5)
    assert [c.as_dict() for c in a] == [c.as_dict() for c in b]
    assert sum(1 for c in a if (c.nx, c.ny, c.nz) == (128, 64, 64)) == 32
    assert sum(1 for c in a if (c.nx, c.ny, c.nz) == (96, 48, 48)) == 32
    assert all(0.08 <= c.cs_unburned <= 0.22 for c in a)
    assert all(0.0 <= c.accel_strength <= 2 * 2.0361 for c in a)
    assert all(0.0 <= c.relax <= 5000.0 for c in a)
    assert len({c.seed for c in a}) == 64
    assert ensemble_configs(64, seed=6)[0].cs_unburned != a[0].cs_unburned
