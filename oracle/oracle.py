"""Python handle on the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers live under ``oracle/``:

* ``liboracle.so`` -- ``les_oracle.c``, a serial plain-C restatement of the reference's
  per-timestep hot path with runtime grid sizes;
* ``_ref/<config>/les_ref`` -- the reference solver itself, compiled by ``build_ref.py``.

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may use this module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import struct
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_ROOT = os.path.join(HERE, "_ref")
DATA_DIR = os.path.join(os.path.dirname(HERE), "combustion-les-optimization_b200", "data")

# field ids (les_oracle.c enum)
FIELD_IDS = {"u": 0, "v": 1, "w": 2, "T": 3, "G": 4, "rho": 5, "Y0": 6, "Y1": 7, "Y2": 8,
             "Y3": 9, "Y4": 10, "nu_t": 11, "S_mag": 12}
_RHS = (["u_f", "v_f", "w_f", "T_f", "G_f", "rho_f"] + [f"Y{k}_f" for k in range(5)]
        + ["nu", "mu_mix", "ST", "Cp", "lambda", "alpha"] + [f"D{k}" for k in range(5)]
        + ["k_rhou", "k_rhov", "k_rhow", "k_T", "k_G"] + [f"k_Y{k}" for k in range(5)])
RHS_IDS = {name: 100 + q for q, name in enumerate(_RHS)}
STATE_NAMES = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]


class OrcConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("num_vortices", C.c_int),
                ("initial_flame_front_i", C.c_int), ("weno_transition_step", C.c_int),
                ("seed", C.c_uint), ("flame_accel", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("inlet_radius", C.c_double), ("rim_outer_radius", C.c_double),
                ("inlet_velocity", C.c_double), ("inlet_temperature", C.c_double),
                ("ambient_temperature", C.c_double), ("turbulence_intensity", C.c_double),
                ("length_scale", C.c_double), ("s_l", C.c_double),
                ("burnt_gas_temperature", C.c_double), ("pr_t", C.c_double), ("sc_t", C.c_double),
                ("d3", C.c_double), ("courant", C.c_double), ("courant_diffusion", C.c_double),
                ("cs_unburned", C.c_double), ("cs_burnt", C.c_double), ("cs_flame_boost", C.c_double),
                ("accel_strength", C.c_double), ("accel_width", C.c_double),
                ("accel_center", C.c_double), ("relax", C.c_double), ("nu_unburnt", C.c_double),
                ("rho_unburnt_approx", C.c_double), ("rho_burnt_approx", C.c_double),
                ("equivalence_ratio", C.c_double)]


def build(quiet: bool = True) -> str:
    """Compile ``les_oracle.c`` into ``liboracle.so`` (same flags as the reference build:
    -O2, no FP contraction)."""
    src = os.path.join(HERE, "les_oracle.c")
    if (os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB_PATH, src, "-lm"]
    subprocess.run(cmd, check=True, capture_output=quiet)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcConfig), C.c_char_p, C.c_char_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_init.argtypes = [C.c_void_p, C.c_int]
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_rhs_only.argtypes = [C.c_void_p, C.c_int]
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_set_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_get_attr.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_dt.restype = C.c_double
        L.orc_dt.argtypes = [C.c_void_p]
        L.orc_t_loop.argtypes = [C.c_void_p]
        L.orc_set_t_loop.argtypes = [C.c_void_p, C.c_int]
        L.orc_max_velocity.restype = C.c_double
        L.orc_max_velocity.argtypes = [C.c_void_p]
        L.orc_get_inflow.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_get_vortices.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_get_inlet_yk.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_sizeof_config.restype = C.c_size_t
        assert L.orc_sizeof_config() == C.sizeof(OrcConfig), "OrcConfig layout mismatch"
        _lib = L
    return _lib


class Oracle:
    """One serial CPU solver instance (the restatement)."""

    def __init__(self, cfg: Dict, chem: Optional[str] = None, tran: Optional[str] = None,
                 start_step: int = 0):
        oc = OrcConfig()
        for name, _t in OrcConfig._fields_:
            setattr(oc, name, cfg[name])
        self.cfg = dict(cfg)
        self.shape = (cfg["nx"], cfg["ny"], cfg["nz"])
        chem = chem or os.path.join(DATA_DIR, "chem.bin")
        tran = tran or os.path.join(DATA_DIR, "tran.bin")
        self._h = lib().orc_create(C.byref(oc), chem.encode(), tran.encode())
        if not self._h:
            raise RuntimeError("orc_create failed (property files?)")
        lib().orc_init(self._h, start_step)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        for _ in range(n):
            lib().orc_step(self._h)

    def rhs_only(self, t_loop: int):
        lib().orc_rhs_only(self._h, t_loop)

    def field(self, name: str) -> np.ndarray:
        fid = FIELD_IDS.get(name, RHS_IDS.get(name))
        out = np.empty(self.shape, dtype=np.float64)
        if lib().orc_get_field(self._h, fid, out.ctypes.data) != 0:
            raise KeyError(name)
        return out

    def set_field(self, name: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.shape
        if lib().orc_set_field(self._h, FIELD_IDS[name], a.ctypes.data) != 0:
            raise KeyError(name)

    def state(self) -> Dict[str, np.ndarray]:
        return {k: self.field(k) for k in STATE_NAMES}

    def attribute(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.int32)
        lib().orc_get_attr(self._h, out.ctypes.data)
        return out

    @property
    def dt(self) -> float:
        return lib().orc_dt(self._h)

    @property
    def t_loop(self) -> int:
        return lib().orc_t_loop(self._h)

    @property
    def max_velocity(self) -> float:
        return lib().orc_max_velocity(self._h)

    def inflow(self) -> np.ndarray:
        ny, nz = self.shape[1], self.shape[2]
        out = np.empty((3, ny, nz), dtype=np.float64)
        lib().orc_get_inflow(self._h, out.ctypes.data)
        return out

    def vortices(self) -> np.ndarray:
        out = np.empty((self.cfg["num_vortices"], 7), dtype=np.float64)
        lib().orc_get_vortices(self._h, out.ctypes.data)
        return out

    def inlet_composition(self):
        a, b, s = (np.empty(5), np.empty(5), np.empty(3))
        lib().orc_get_inlet_yk(self._h, a.ctypes.data, b.ctypes.data, s.ctypes.data)
        return a, b, s


# ------------------------------------------------------------------ compiled reference

def ref_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_ROOT, name, "les_ref"))


def run_reference(name: str, steps: int, seed: int = 1234, start: int = 0, dump_every: int = 1,
                  rhs_dump_step: int = -1, threads: int = 1, env_extra: Optional[Dict] = None,
                  keep_dir: Optional[str] = None, novtk: bool = True, timeout: float = 3600.0,
                  binary: Optional[str] = None, resume: bool = False):
    """Run the compiled reference for ``steps`` steps in a scratch directory.

    ``binary`` runs another build of the same grid instead (the reference with the GPU
    drop-in spliced into its loop, tests/dropin/build_dropin.py); it reads the same
    environment and writes the same files.  ``resume`` keeps an existing restart_info.txt in
    ``keep_dir``, so the reference auto-resumes from the checkpoint there (:4150-4193).

    Returns ``(dumps, meta)``: ``dumps[n]`` is the state after ``n`` steps (dict of
    arrays + 'dt'), ``meta`` holds the per-step wall times, probe CSV texts and the monitor
    CSV text.
    """
    from build_ref import CONFIGS, STATE_FIELDS, RHS1_FIELDS  # noqa: local module
    cfg = CONFIGS[name]
    exe = binary or os.path.join(REF_ROOT, name, "les_ref")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    work = keep_dir or tempfile.mkdtemp(prefix=f"lesref_{name}_")
    os.makedirs(work, exist_ok=True)
    for fn in ("chem.bin", "tran.bin"):
        shutil.copyfile(os.path.join(REF_ROOT, name, fn), os.path.join(work, fn))
    rinfo = os.path.join(work, "restart_info.txt")
    if os.path.exists(rinfo) and not resume:
        os.remove(rinfo)          # the reference auto-resumes when this file exists
    env = dict(os.environ)
    env.update({"OMP_NUM_THREADS": str(threads), "LES_REF_STEPS": str(steps),
                "LES_REF_SEED": str(seed), "LES_REF_START": str(start),
                "LES_REF_DUMP_EVERY": str(dump_every), "LES_REF_RHS_DUMP_STEP": str(rhs_dump_step),
                "LES_REF_NOVTK": "1" if novtk else "0"})
    if env_extra:
        env.update({k: str(v) for k, v in env_extra.items()})
    p = subprocess.run([exe], cwd=work, env=env, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference failed rc={p.returncode}: {p.stderr[-2000:]}")
    shape = (cfg["nx"], cfg["ny"], cfg["nz"])
    ncell = shape[0] * shape[1] * shape[2]
    dumps = {}
    if dump_every > 0:
        wanted = sorted(set(range(dump_every, steps + 1, dump_every))
                        | ({1} if os.path.exists(os.path.join(work, "state_000001.bin")) else set()))
        for n in wanted:
            path = os.path.join(work, f"state_{n:06d}.bin")
            with open(path, "rb") as f:
                raw = f.read()
            t, = struct.unpack_from("<i", raw, 0)
            dt, = struct.unpack_from("<d", raw, 4)
            arr = np.frombuffer(raw, dtype=np.float64, offset=12).reshape(len(STATE_FIELDS), *shape)
            d = {k: arr[q].copy() for q, k in enumerate(STATE_FIELDS)}
            d["dt"] = dt
            d["t"] = t
            dumps[n] = d
    rhs1 = None
    rp = os.path.join(work, "rhs1.bin")
    if rhs_dump_step >= 0 and os.path.exists(rp):
        arr = np.fromfile(rp, dtype=np.float64).reshape(len(RHS1_FIELDS), *shape)
        rhs1 = {k: arr[q].copy() for q, k in enumerate(RHS1_FIELDS)}
    times = []
    for line in p.stderr.splitlines():
        if line.startswith("LESREF_STEP"):
            _, t, dt, wall = line.split()
            times.append((int(t), float(dt), float(wall)))
    probes = {}
    for n in range(7):
        pp = os.path.join(work, f"probe_data_flame_region_loc{n}.csv")
        if os.path.exists(pp):
            with open(pp) as f:
                probes[n] = f.read()
    mon = ""
    mp = os.path.join(work, "simulation_monitor.csv")
    if os.path.exists(mp):
        with open(mp) as f:
            mon = f.read()
    meta = {"times": times, "probes": probes, "monitor": mon, "rhs1": rhs1, "dir": work,
            "stdout": p.stdout}
    if keep_dir is None:
        shutil.rmtree(work, ignore_errors=True)
    return dumps, meta
