"""End of run and resume (les_solver_finish / les_solver_resume) on the CPU: the host driver
host/les_host.c linked against a stand-in for the CUDA library (tests/solver_fake/fake_gpu.c),
whose step depends on dt, t_loop, the vortex table, the inflow noise and the attribute map.

* LES_RESUME_REFERENCE keeps the reference's resume defects (les_combustion_solver.c:4623,
  :4138-4193): checkpoint and restart_info at step 0, rand() re-seeded and the vortices
  redrawn, the start-up attribute map without the j = 0 symmetry code, nu/alpha maxima 0.
* LES_RESUME_FIXED continues the uninterrupted run exactly.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

REFERENCE, FIXED = 0, 1


@pytest.fixture(scope="module")
def L(tmp_path_factory):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    out = str(tmp_path_factory.mktemp("fakesolver") / "libfakesolver.so")
    subprocess.run([gcc, "-shared", "-fPIC", "-O1", "-std=c11", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(PKG, "host"), os.path.join(PKG, "host", "les_host.c"),
                    os.path.join(ROOT, "tests", "solver_fake", "fake_gpu.c"), "-o", out, "-lm"], check=True)
    lib = C.CDLL(out)
    vp = C.c_void_p
    lib.les_solver_create.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(vp)]
    lib.les_solver_run.argtypes = [vp, C.c_int]
    lib.les_solver_finish.argtypes = [vp, C.c_char_p, C.c_int]
    lib.les_solver_resume.argtypes = [vp, C.c_char_p, C.c_int, C.POINTER(C.c_int)]
    lib.les_solver_t_loop.argtypes = [vp]
    lib.les_solver_last_dt.argtypes = [vp]
    lib.les_solver_last_dt.restype = C.c_double
    lib.les_solver_vortices.argtypes = [vp, vp]
    lib.les_solver_rng_draws.argtypes = [vp]
    lib.les_solver_rng_draws.restype = C.c_ulonglong
    lib.les_solver_attribute.argtypes = [vp, vp]
    lib.les_solver_ctx.argtypes = [vp]
    lib.les_solver_ctx.restype = vp
    lib.les_solver_destroy.argtypes = [vp]
    lib.lesgpu_download_state.argtypes = [vp, C.POINTER(vp), C.c_int]
    lib.lesgpu_dt_inputs.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.fake_attr.argtypes = [vp, vp]
    return lib


class Sol:
    def __init__(self, L):
        from lesgpu.config import preset
        from lesgpu.native import LesgpuConfig
        self.L = L
        self.cfg = preset("tiny", seed=321)
        self.c = LesgpuConfig.from_config(self.cfg)
        self.h = C.c_void_p()
        assert L.les_solver_create(C.byref(self.c), b"unused", b"unused", 0, C.byref(self.h)) == 0
        self.shape = (self.cfg.nx, self.cfg.ny, self.cfg.nz)

    def run(self, n):
        assert self.L.les_solver_run(self.h, n) == 0

    def state(self):
        arrs = [np.empty(self.shape) for _ in range(11)]
        ptrs = (C.c_void_p * 11)(*[a.ctypes.data for a in arrs])
        assert self.L.lesgpu_download_state(self.L.les_solver_ctx(self.h), ptrs, 11) == 0
        return arrs

    def vortices(self):
        v = np.empty((self.cfg.num_vortices, 7))
        self.L.les_solver_vortices(self.h, v.ctypes.data)
        return v

    def attribute(self):
        a = np.empty(self.shape, dtype=np.int32)
        self.L.les_solver_attribute(self.h, a.ctypes.data)
        d = np.empty(self.shape, dtype=np.int32)
        uploads = self.L.fake_attr(self.L.les_solver_ctx(self.h), d.ctypes.data)
        return a, d, uploads

    def dt_inputs(self):
        u, n, a = C.c_double(), C.c_double(), C.c_double()
        self.L.lesgpu_dt_inputs(self.L.les_solver_ctx(self.h), C.byref(u), C.byref(n), C.byref(a))
        return u.value, n.value, a.value

    def t(self):
        return self.L.les_solver_t_loop(self.h)

    def close(self):
        self.L.les_solver_destroy(self.h)


def test_reference_mode_keeps_the_reference_defects(L, tmp_path):
    a = Sol(L)
    a.run(7)
    assert a.t() == 7
    d = str(tmp_path).encode()
    assert L.les_solver_finish(a.h, d, REFERENCE) == 0
    raw = np.fromfile(tmp_path / "checkpoint.bin", dtype=np.uint8)
    assert int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0]) == 0          # save_quick_checkpoint(0)
    assert (tmp_path / "restart_info.txt").read_text() == "BINARY\n0\n"
    assert not (tmp_path / "les_resume.bin").exists()
    st_a = a.state()
    fresh = Sol(L)
    b = Sol(L)
    b.run(3)                                    # a solver that has moved on before resuming
    t = C.c_int(-1)
    assert L.les_solver_resume(b.h, d, REFERENCE, C.byref(t)) == 0
    assert t.value == 0 and b.t() == 0          # the step count starts again
    for x, y in zip(b.state(), st_a):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(b.vortices(), fresh.vortices())      # vortices redrawn from the seed
    assert L.les_solver_rng_draws(b.h) == L.les_solver_rng_draws(fresh.h) == 3 + 7 * a.cfg.num_vortices
    attr_host, attr_dev, uploads = b.attribute()
    attr0, _, _ = fresh.attribute()
    assert (attr0[1:-1, 0, :] == 5).any()
    want = attr0.copy()
    want[(want == 5) | (want == 6)] = 4                                # the start-up map (:4123-4136)
    np.testing.assert_array_equal(attr_host, want)
    np.testing.assert_array_equal(attr_dev, want)
    assert uploads == 2
    assert b.dt_inputs()[1:] == (0.0, 0.0)                             # nu/alpha maxima not restored
    for s in (a, b, fresh):
        s.close()


def test_fixed_mode_continues_the_run_exactly(L, tmp_path):
    d = str(tmp_path).encode()
    a = Sol(L)
    a.run(7)
    assert L.les_solver_finish(a.h, d, FIXED) == 0
    raw = np.fromfile(tmp_path / "checkpoint.bin", dtype=np.uint8)
    assert int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0]) == 7
    assert (tmp_path / "restart_info.txt").read_text() == "BINARY\n7\n"
    assert (tmp_path / "les_resume.bin").exists()
    a.run(5)
    b = Sol(L)
    t = C.c_int(-1)
    assert L.les_solver_resume(b.h, d, FIXED, C.byref(t)) == 0
    assert t.value == 7
    b.run(5)
    assert a.t() == b.t() == 12
    assert L.les_solver_last_dt(a.h) == L.les_solver_last_dt(b.h)
    assert L.les_solver_rng_draws(a.h) != 0
    np.testing.assert_array_equal(a.vortices(), b.vortices())
    for x, y in zip(a.state(), b.state()):
        np.testing.assert_array_equal(x, y)
    attr_a, _, _ = a.attribute()
    attr_b, dev_b, uploads = b.attribute()
    np.testing.assert_array_equal(attr_a, attr_b)                      # setting()'s map kept
    assert uploads == 1
    assert a.dt_inputs() == b.dt_inputs()
    # a reference-mode resume of the same files differs: its first dt has no diffusion limit
    c = Sol(L)
    assert L.les_solver_resume(c.h, d, REFERENCE, C.byref(t)) == 0
    assert t.value == 7
    c.run(1)
    a2 = Sol(L)
    assert L.les_solver_resume(a2.h, d, FIXED, C.byref(t)) == 0
    a2.run(1)
    assert L.les_solver_last_dt(c.h) > L.les_solver_last_dt(a2.h)
    for s in (a, b, c, a2):
        s.close()


def test_resume_errors(L, tmp_path):
    a = Sol(L)
    t = C.c_int(-1)
    assert L.les_solver_resume(a.h, str(tmp_path).encode(), REFERENCE, C.byref(t)) == -4     # no restart_info.txt
    a.run(2)
    assert L.les_solver_finish(a.h, str(tmp_path).encode(), REFERENCE) == 0
    assert L.les_solver_resume(a.h, str(tmp_path).encode(), FIXED, C.byref(t)) == -4         # no sidecar
    assert L.les_solver_resume(a.h, str(tmp_path).encode(), 7, C.byref(t)) == -1             # unknown mode
    (tmp_path / "restart_info.txt").write_text("results.vtk\n40\n")
    assert L.les_solver_resume(a.h, str(tmp_path).encode(), REFERENCE, C.byref(t)) == -4     # VTK restarts: not built
    a.close()
