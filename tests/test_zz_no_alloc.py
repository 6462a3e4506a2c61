"""lesgpu_monitor_noalloc: the allocation-free monitor entry point, for callers that may
not allocate device memory (memory-budgeted serving loops, latency-bound paths that must
not take cudaMalloc's synchronisation).

Called through the C ABI on caller-owned device buffers, twice in a row on the same
scratch array, and compared with lesgpu_monitor (the allocating entry point) on the same
state, then on ragged sizes (a partial last block, and fewer blocks than the call before)
against numpy on the first n cells.  The mass sum is reduced in a different order, so it is
compared to 1e-13 relative; the minima and maxima are exact.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_monitor_noalloc_matches_monitor(lesgpu_native, cuda_device):
    import torch
    from lesgpu.config import preset
    N = lesgpu_native
    L = N.lib()
    fn = L.lesgpu_monitor_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_size_t, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_void_p, ctypes.c_void_p]
    cfg = preset("c1")
    sol = N.Solver(cfg)
    dx, dy, dz = cfg.lx / cfg.nx, cfg.ly / cfg.ny, cfg.lz / cfg.nz
    for call in range(2):
        sol.step(2)
        want = sol.ctx.monitor()
        st = sol.state()
        dev = {k: torch.from_numpy(np.ascontiguousarray(st[k])).to("cuda:0") for k in ("rho", "T", "G", "Y0")}
        out = torch.full((6,), float("nan"), dtype=torch.float64, device="cuda:0")
        stream = torch.cuda.current_stream().cuda_stream
        rc = fn(dev["rho"].data_ptr(), dev["T"].data_ptr(), dev["G"].data_ptr(), dev["Y0"].data_ptr(), cfg.cells,
                dx, dy, dz, out.data_ptr(), stream)
        assert rc == 0, f"call {call}: rc {rc}"
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert abs(got[0] - want[0]) <= 1e-13 * abs(want[0]), (call, got[0], want[0])
        np.testing.assert_array_equal(got[1:], want[1:])
    # ragged sizes on the same arrays: a partial last block, then fewer blocks than the call
    # before (the per-block partials are laid out by the current call's block count)
    flat = {k: np.ascontiguousarray(st[k]).ravel() for k in ("rho", "T", "G", "Y0")}
    for n in (cfg.cells - 37, 1000 + 5):
        out.fill_(float("nan"))
        rc = fn(dev["rho"].data_ptr(), dev["T"].data_ptr(), dev["G"].data_ptr(), dev["Y0"].data_ptr(), n,
                dx, dy, dz, out.data_ptr(), stream)
        assert rc == 0, f"n={n}: rc {rc}"
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        mass = float(np.sum(((flat["rho"][:n] * dx) * dy) * dz))
        assert abs(got[0] - mass) <= 1e-13 * abs(mass), (n, got[0], mass)
        want_n = [flat["T"][:n].min(), flat["T"][:n].max(), flat["G"][:n].min(), flat["G"][:n].max(),
                  flat["Y0"][:n].min()]
        np.testing.assert_array_equal(got[1:], want_n)
    # an output buffer in host memory is refused before anything is launched
    host_out = np.zeros(6)
    assert fn(dev["rho"].data_ptr(), dev["T"].data_ptr(), dev["G"].data_ptr(), dev["Y0"].data_ptr(), cfg.cells,
              dx, dy, dz, host_out.ctypes.data, stream) == -1
    too_big = N.lib().lesgpu_monitor_noalloc(dev["rho"].data_ptr(), dev["T"].data_ptr(), dev["G"].data_ptr(),
                                             dev["Y0"].data_ptr(), 16777216 + 1, dx, dy, dz, out.data_ptr(), stream)
    assert too_big == -1
    sol.close()
