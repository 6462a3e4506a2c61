"""The C-ABI library loads on a CPU-only machine and exports every entry point that
include/*.h declares (no compute calls are made here)."""
import ctypes
import glob
import os
import re

from conftest import ROOT

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b((?:lesgpu|les)_\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        with open(h) as f:
            txt = f.read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in DECL.finditer(txt):
            names.add(m.group(1))
    return names


def test_headers_declare_the_boundary():
    names = declared_functions()
    for want in ["lesgpu_create", "lesgpu_upload_state", "lesgpu_dt_inputs", "lesgpu_set_inflow", "lesgpu_step",
                 "lesgpu_probe_lines", "lesgpu_monitor", "lesgpu_download_state", "lesgpu_last_error",
                 "lesgpu_destroy", "les_solver_create", "les_solver_step", "les_rng_next"]:
        assert want in names


def test_library_exports_every_declared_symbol(lesgpu_native):
    lib = ctypes.CDLL(lesgpu_native.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from lesgpu import native
    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", str(tmp_path / "liblesgpu.so"))
    try:
        native.lib()
    except FileNotFoundError as e:
        assert "build.py" in str(e)
    else:
        raise AssertionError("expected FileNotFoundError")


def test_bind_device_rejects_a_negative_device(lesgpu_native):
    lib = ctypes.CDLL(lesgpu_native.LIB_PATH)
    lib.lesgpu_bind_device.argtypes = [ctypes.c_int]
    lib.lesgpu_bind_device.restype = ctypes.c_int
    assert lib.lesgpu_bind_device(-1) == -1          # LESGPU_EINVAL, no CUDA call made


def test_tile_tables_agree():
    """The tile table of the kernels (csrc/les_ctx.h), the count the header publishes
    (LESGPU_NTILES: lesgpu_autotune writes 4 x LESGPU_NTILES times into the caller's buffer)
    and the binding's table, which sizes that buffer, list the same tiles."""
    from lesgpu import native
    with open(os.path.join(ROOT, "include", "les_gpu.h")) as f:
        ntiles = int(re.search(r"#define\s+LESGPU_NTILES\s+(\d+)", f.read()).group(1))
    with open(os.path.join(ROOT, "combustion-les-optimization_b200", "csrc", "les_ctx.h")) as f:
        ctx = f.read()
    body = re.search(r"kShapes\[NSHAPES\]\s*=\s*\{(.*?)\};", ctx, re.S).group(1)
    shapes = [tuple(int(x) for x in m) for m in re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*\}", body)]
    assert int(re.search(r"constexpr int NSHAPES = (\d+);", ctx).group(1)) == ntiles
    assert len(shapes) == ntiles
    assert [tuple(t) for t in native.Context.TILES] == shapes
    n256 = int(re.search(r"constexpr int NSHAPES_256 = (\d+);", ctx).group(1))
    assert all(bx * by * bz == 256 for bx, by, bz in shapes[:n256])
    assert all(bx * by * bz == 512 for bx, by, bz in shapes[n256:])
