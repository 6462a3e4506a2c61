"""ctypes binding of ``liblesgpu.so`` (include/les_gpu.h and include/les_solver.h).

The library is built in-tree by ``build.py``.  There is no fallback: if the shared
library is missing or a CUDA call fails, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

from .config import SolverConfig

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# LESGPU_LIB selects another build of the same library (tuning variants); default in-tree.
LIB_PATH = os.environ.get("LESGPU_LIB") or os.path.join(PKG_DIR, "liblesgpu.so")
DATA_DIR = os.path.join(PKG_DIR, "data")
CHEM_BIN = os.path.join(DATA_DIR, "chem.bin")
TRAN_BIN = os.path.join(DATA_DIR, "tran.bin")

FP64, FP32 = 0, 1
STATE_NAMES = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4"]
FIELD_IDS: Dict[str, int] = {name: q for q, name in enumerate(STATE_NAMES)}
FIELD_IDS.update({"nu_t": 11, "S_mag": 12})
_INSPECT = (["u_f", "v_f", "w_f", "T_f", "G_f", "rho_f"] + [f"Y{k}_f" for k in range(5)]
            + ["nu", "mu_mix", "ST", "Cp", "lambda", "alpha"] + [f"D{k}" for k in range(5)]
            + ["k_rhou", "k_rhov", "k_rhow", "k_T", "k_G"] + [f"k_Y{k}" for k in range(5)])
FIELD_IDS.update({name: 100 + q for q, name in enumerate(_INSPECT)})

ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "EIO", -5: "ESTATE", -6: "ENONFINITE"}
LESGPU_EINVAL, LESGPU_ECUDA, LESGPU_ENOMEM, LESGPU_EIO, LESGPU_ESTATE, LESGPU_ENONFINITE = -1, -2, -3, -4, -5, -6

LES_OUT_PROBES, LES_OUT_MONITOR, LES_OUT_CHECKPOINT, LES_OUT_POINTS, LES_OUT_VTK = 1, 2, 4, 8, 16
LES_OUT_PSTAT = 32          # probe-row statistics on the device -> profile_stats.bin
AVG_NAMES = ["u", "v", "w", "uu", "vv", "ww", "uv", "uw", "vw", "G"]
STRESS_NAMES = ["uu", "vv", "ww", "uv", "uw", "vw", "G_mean"]


# les_solver_finish / les_solver_resume modes (les_solver.h)
RESUME_REFERENCE = 0
RESUME_FIXED = 1


class LesgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class LesgpuConfig(C.Structure):
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
                ("equivalence_ratio", C.c_double), ("precision", C.c_int), ("device", C.c_int)]

    @classmethod
    def from_config(cls, cfg: SolverConfig, precision: int = FP64, device: int = 0) -> "LesgpuConfig":
        c = cls()
        d = cfg.as_dict()
        for name, _t in cls._fields_:
            if name in d:
                setattr(c, name, d[name])
        c.precision = precision
        c.device = device
        return c


class LesgpuSpecies(C.Structure):
    _fields_ = [("mw", C.c_double * 5), ("t_mid", C.c_double * 5),
                ("nasa_high", (C.c_double * 7) * 5), ("nasa_low", (C.c_double * 7) * 5),
                ("lam", (C.c_double * 4) * 5), ("eta", (C.c_double * 4) * 5),
                ("dcoef", ((C.c_double * 4) * 5) * 5)]


class LesRng(C.Structure):
    _fields_ = [("r", C.c_int * 34), ("f", C.c_int), ("b", C.c_int), ("n", C.c_ulonglong)]


_lib = None


def _sig(L, name, res, args):
    fn = getattr(L, name)
    fn.restype = res
    fn.argtypes = args


def lib():
    """Load ``liblesgpu.so``; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python build.py` in {PKG_DIR}")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.c_void_p
        _sig(L, "lesgpu_load_species", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(LesgpuSpecies)])
        _sig(L, "lesgpu_create", C.c_int, [C.POINTER(LesgpuConfig), C.POINTER(LesgpuSpecies), C.POINTER(vp)])
        _sig(L, "lesgpu_destroy", None, [vp])
        _sig(L, "lesgpu_last_error", C.c_char_p, [vp])
        _sig(L, "lesgpu_upload_attribute", C.c_int, [vp, vp])
        _sig(L, "lesgpu_upload_state", C.c_int, [vp, C.POINTER(C.c_void_p), C.c_int])
        _sig(L, "lesgpu_download_state", C.c_int, [vp, C.POINTER(C.c_void_p), C.c_int])
        _sig(L, "lesgpu_get_field", C.c_int, [vp, C.c_int, dp])
        _sig(L, "lesgpu_dt_inputs", C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                               C.POINTER(C.c_double)])
        _sig(L, "lesgpu_set_inflow", C.c_int, [vp, dp, C.c_int, dp])
        _sig(L, "lesgpu_step", C.c_int, [vp, C.c_double, C.c_int])
        _sig(L, "lesgpu_probe_lines", C.c_int, [vp, vp, C.c_int, C.c_int, dp])
        _sig(L, "lesgpu_monitor", C.c_int, [vp, dp])
        _sig(L, "lesgpu_check_finite", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_set_debug", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_eval_rhs", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_sync", C.c_int, [vp])
        _sig(L, "lesgpu_kernel_timing", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_kernel_times", C.c_int, [vp, dp, dp, C.c_int])
        _sig(L, "lesgpu_mark", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_selfcheck_division", C.c_int, [dp, C.c_int, C.c_size_t, C.c_ulonglong,
                                                       C.POINTER(C.c_ulonglong)])
        _sig(L, "lesgpu_elapsed_ms", C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_double)])
        _sig(L, "lesgpu_device_bytes", C.c_size_t, [vp])
        _sig(L, "lesgpu_bytes_for_grid", C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int])
        _sig(L, "les_rng_seed", None, [C.POINTER(LesRng), C.c_uint])
        _sig(L, "les_rng_next", C.c_int, [C.POINTER(LesRng)])
        _sig(L, "les_initial_state", C.c_int, [C.POINTER(LesgpuConfig), C.POINTER(LesgpuSpecies), vp,
                                               C.POINTER(C.c_void_p)])
        _sig(L, "les_vortices_init", None, [C.POINTER(LesRng), C.POINTER(LesgpuConfig), dp])
        _sig(L, "les_vortices_update", None, [C.POINTER(LesRng), C.POINTER(LesgpuConfig), dp, C.c_double])
        _sig(L, "les_inflow_noise", None, [C.POINTER(LesRng), vp, C.c_int, C.c_int, dp])
        _sig(L, "les_dt", C.c_double, [C.POINTER(LesgpuConfig), C.c_double, C.c_double, C.c_double])
        _sig(L, "les_solver_create", C.c_int, [C.POINTER(LesgpuConfig), C.c_char_p, C.c_char_p, C.c_int,
                                               C.POINTER(vp)])
        _sig(L, "les_solver_destroy", None, [vp])
        _sig(L, "les_solver_ctx", vp, [vp])
        _sig(L, "les_solver_last_error", C.c_char_p, [vp])
        _sig(L, "les_solver_set_outputs", C.c_int, [vp, C.c_char_p, C.c_int])
        _sig(L, "les_solver_step", C.c_int, [vp])
        _sig(L, "les_solver_run", C.c_int, [vp, C.c_int])
        _sig(L, "les_solver_run_device", C.c_int, [vp, C.c_int, C.c_int])
        _sig(L, "les_solver_loop_begin", C.c_int, [vp, C.c_int])
        _sig(L, "les_solver_loop_run", C.c_int, [vp, C.c_int])
        _sig(L, "les_solver_loop_end", C.c_int, [vp])
        _sig(L, "les_solver_next_chunk", C.c_int, [vp, C.c_int])
        _sig(L, "les_solver_set_averaging", C.c_int, [vp, C.c_int])
        _sig(L, "les_solver_save_stats", C.c_int, [vp, C.c_char_p])
        _sig(L, "les_solver_load_stats", C.c_int, [vp, C.c_char_p])
        _sig(L, "les_solver_reynolds_stresses", C.c_int, [vp, vp, C.POINTER(C.c_int)])
        _sig(L, "les_solver_flush", C.c_int, [vp])
        _sig(L, "lesgpu_avg_begin", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_avg_end", C.c_int, [vp])
        _sig(L, "lesgpu_avg_download", C.c_int, [vp, vp, C.POINTER(C.c_int)])
        _sig(L, "lesgpu_avg_upload", C.c_int, [vp, vp, C.c_int])
        _sig(L, "les_solver_loop_collect", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_autotune", C.c_int, [vp, C.c_int, vp, dp])
        _sig(L, "lesgpu_set_scalar_staging", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_get_scalar_staging", C.c_int, [vp])
        _sig(L, "lesgpu_set_tiles", C.c_int, [vp, vp])
        _sig(L, "lesgpu_get_tiles", C.c_int, [vp, vp])
        _sig(L, "lesgpu_group_create", C.c_int, [vp, C.c_int, C.POINTER(vp)])
        _sig(L, "lesgpu_group_run", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_group_destroy", None, [vp])
        _sig(L, "les_ensemble_create", C.c_int, [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(vp)])
        _sig(L, "les_ensemble_run", C.c_int, [vp, C.c_int, C.c_int])
        _sig(L, "les_ensemble_set_batched", C.c_int, [vp, C.c_int, C.c_int])
        _sig(L, "lesgpu_group_create_batched", C.c_int, [vp, C.c_int, C.c_int, C.POINTER(vp)])
        _sig(L, "lesgpu_group_batches", C.c_int, [vp])
        _sig(L, "les_ensemble_size", C.c_int, [vp])
        _sig(L, "les_ensemble_member", vp, [vp, C.c_int])
        _sig(L, "les_ensemble_last_error", C.c_char_p, [vp])
        _sig(L, "les_ensemble_destroy", None, [vp])
        _sig(L, "lesgpu_loop_begin", C.c_int, [vp, vp, dp, C.c_int, C.c_int])
        _sig(L, "lesgpu_loop_config", C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int])
        _sig(L, "lesgpu_run", C.c_int, [vp, C.c_int])
        _sig(L, "lesgpu_loop_history", C.c_int, [vp, C.c_int, dp, dp, dp, dp])
        _sig(L, "lesgpu_loop_end", C.c_int, [vp, vp, dp, C.POINTER(C.c_int)])
        _sig(L, "les_solver_t_loop", C.c_int, [vp])
        _sig(L, "les_solver_last_dt", C.c_double, [vp])
        _sig(L, "les_solver_last_umax", C.c_double, [vp])
        _sig(L, "les_solver_attribute", C.c_int, [vp, vp])
        _sig(L, "les_solver_save_checkpoint", C.c_int, [vp, C.c_char_p, C.c_int])
        _sig(L, "les_solver_load_checkpoint", C.c_int, [vp, C.c_char_p, C.POINTER(C.c_int)])
        _sig(L, "les_solver_vortices", C.c_int, [vp, dp])
        _sig(L, "les_solver_rng_draws", C.c_ulonglong, [vp])
        _sig(L, "les_solver_finish", C.c_int, [vp, C.c_char_p, C.c_int])
        _sig(L, "les_solver_resume", C.c_int, [vp, C.c_char_p, C.c_int, C.POINTER(C.c_int)])
        _sig(L, "lesgpu_set_dt_inputs", C.c_int, [vp, C.c_double, C.c_double])
        _sig(L, "les_solver_pstat_begin", C.c_int, [vp, dp, C.c_int, dp, C.c_int, dp, C.c_int, dp, dp, C.c_int])
        _sig(L, "les_solver_pstat_size", C.c_size_t, [vp])
        _sig(L, "les_solver_pstat_read", C.c_int, [vp, dp])
        _lib = L
    return _lib


def load_species(chem: str = CHEM_BIN, tran: str = TRAN_BIN) -> LesgpuSpecies:
    sp = LesgpuSpecies()
    rc = lib().lesgpu_load_species(chem.encode(), tran.encode(), C.byref(sp))
    if rc != 0:
        raise LesgpuError(rc, f"cannot load species from {chem}, {tran}")
    return sp


def _ptrs(arrs: Sequence[np.ndarray]):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class Rng:
    """The glibc rand() stream (srand/rand) with private state."""

    def __init__(self, seed: int):
        self._s = LesRng()
        lib().les_rng_seed(C.byref(self._s), seed)

    def next(self) -> int:
        return lib().les_rng_next(C.byref(self._s))

    @property
    def draws(self) -> int:
        return self._s.n


def selfcheck_division(divisors: Sequence[float], n: int, seed: int = 12345) -> int:
    """Number of quotients where the kernels' constant division differs from IEEE division."""
    d = np.ascontiguousarray(divisors, dtype=np.float64)
    bad = C.c_ulonglong(0)
    rc = lib().lesgpu_selfcheck_division(d.ctypes.data, len(d), n, seed, C.byref(bad))
    if rc != 0:
        raise LesgpuError(rc, "selfcheck_division")
    return int(bad.value)


def initial_state(cfg: SolverConfig, species: Optional[LesgpuSpecies] = None):
    """Attribute map and state of a fresh run (the reference's initialize()+setting())."""
    sp = species or load_species()
    shape = (cfg.nx, cfg.ny, cfg.nz)
    attr = np.empty(shape, dtype=np.int32)
    fields = [np.empty(shape, dtype=np.float64) for _ in STATE_NAMES]
    c = LesgpuConfig.from_config(cfg)
    rc = lib().les_initial_state(C.byref(c), C.byref(sp), attr.ctypes.data, _ptrs(fields))
    if rc != 0:
        raise LesgpuError(rc, "les_initial_state")
    return attr, dict(zip(STATE_NAMES, fields))


class Context:
    """One ``lesgpu_ctx``: device arena of one grid driven through the C ABI."""

    def __init__(self, cfg: SolverConfig, precision: int = FP64, species: Optional[LesgpuSpecies] = None,
                 device: int = 0):
        self.cfg = cfg
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self._sp = species or load_species()
        self._c = LesgpuConfig.from_config(cfg, precision, device)
        h = C.c_void_p()
        rc = lib().lesgpu_create(C.byref(self._c), C.byref(self._sp), C.byref(h))
        if rc != 0:
            raise LesgpuError(rc, "lesgpu_create failed")
        self._h = h

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise LesgpuError(rc, f"{what}: {lib().lesgpu_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            lib().lesgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_attribute(self, attr: np.ndarray):
        a = np.ascontiguousarray(attr, dtype=np.int32)
        assert a.shape == self.shape
        self._check(lib().lesgpu_upload_attribute(self._h, a.ctypes.data), "upload_attribute")

    def upload_state(self, state: Dict[str, np.ndarray]):
        arrs = [np.ascontiguousarray(state[k], dtype=np.float64) for k in STATE_NAMES]
        for a in arrs:
            assert a.shape == self.shape
        self._check(lib().lesgpu_upload_state(self._h, _ptrs(arrs), len(arrs)), "upload_state")

    def download_state(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """The state Phi_n as float64 host arrays; ``out`` (C-contiguous float64 arrays of the
        grid's shape, e.g. views of pinned buffers) receives it in place."""
        if out is None:
            arrs = [np.empty(self.shape, dtype=np.float64) for _ in STATE_NAMES]
        else:
            arrs = [out[k] for k in STATE_NAMES]
            for a in arrs:
                if a.dtype != np.float64 or a.shape != self.shape or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError("download_state: out arrays must be writeable C-contiguous float64 of the grid shape")
        self._check(lib().lesgpu_download_state(self._h, _ptrs(arrs), len(arrs)), "download_state")
        return dict(zip(STATE_NAMES, arrs))

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(lib().lesgpu_get_field(self._h, FIELD_IDS[name], out.ctypes.data), f"get_field({name})")
        return out

    def dt_inputs(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._check(lib().lesgpu_dt_inputs(self._h, C.byref(a), C.byref(b), C.byref(c)), "dt_inputs")
        return a.value, b.value, c.value

    def set_inflow(self, vortices: np.ndarray, noise: np.ndarray):
        v = np.ascontiguousarray(vortices, dtype=np.float64)
        n = np.ascontiguousarray(noise, dtype=np.float64)
        self._check(lib().lesgpu_set_inflow(self._h, v.ctypes.data, v.shape[0], n.ctypes.data), "set_inflow")

    def step(self, dt: float, t_loop: int):
        self._check(lib().lesgpu_step(self._h, dt, t_loop), "step")

    def eval_rhs(self, t_loop: int):
        self._check(lib().lesgpu_eval_rhs(self._h, t_loop), "eval_rhs")

    def set_debug(self, on: bool = True):
        self._check(lib().lesgpu_set_debug(self._h, 1 if on else 0), "set_debug")

    def probe_lines(self, stations: Sequence[int], k_line: int) -> np.ndarray:
        st = np.ascontiguousarray(stations, dtype=np.int32)
        out = np.empty((len(st), self.shape[1], 6), dtype=np.float64)
        self._check(lib().lesgpu_probe_lines(self._h, st.ctypes.data, len(st), k_line, out.ctypes.data),
                    "probe_lines")
        return out

    def monitor(self) -> np.ndarray:
        out = np.empty(6, dtype=np.float64)
        self._check(lib().lesgpu_monitor(self._h, out.ctypes.data), "monitor")
        return out

    def check_finite(self, name: str = "u") -> bool:
        rc = lib().lesgpu_check_finite(self._h, FIELD_IDS[name])
        if rc == -6:
            return False
        self._check(rc, "check_finite")
        return True

    def sync(self):
        self._check(lib().lesgpu_sync(self._h), "sync")

    def mark(self, slot: int):
        self._check(lib().lesgpu_mark(self._h, slot), "mark")

    def elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_double()
        self._check(lib().lesgpu_elapsed_ms(self._h, a, b, C.byref(v)), "elapsed_ms")
        return v.value

    # thread-block tiles (k extent, j extent, i extent) indexed by lesgpu_set_tiles, per
    # class {filter, strain, rhs_flow, rhs_scalar, eos}; the 512-thread tiles from index 8 on
    # serve the strain, flow and scalar classes only (LESGPU_NTILES entries in all)
    TILES = [(32, 8, 1), (64, 4, 1), (16, 16, 1), (128, 2, 1), (32, 4, 2), (16, 8, 2), (32, 2, 4), (16, 4, 4),
             (32, 8, 2), (32, 4, 4), (16, 8, 4), (16, 4, 8), (64, 4, 2)]

    def autotune(self, reps: int = 3):
        """Install the fastest tile per kernel class; returns (tiles[5], ms[4 classes, tiles])."""
        nt = len(self.TILES)
        tiles = np.zeros(5, dtype=np.int32)
        ms = np.zeros(4 * nt)
        self._check(lib().lesgpu_autotune(self._h, reps, tiles.ctypes.data, ms.ctypes.data), "autotune")
        return tiles.tolist(), ms.reshape(4, nt)

    def set_tiles(self, tiles):
        t = np.ascontiguousarray(tiles, dtype=np.int32)
        self._check(lib().lesgpu_set_tiles(self._h, t.ctypes.data), "set_tiles")

    def set_scalar_staging(self, enable: bool):
        """The scalar pass with TMA-staged stencil fields (same arithmetic, same bits)."""
        self._check(lib().lesgpu_set_scalar_staging(self._h, 1 if enable else 0), "set_scalar_staging")

    def get_scalar_staging(self) -> bool:
        return bool(lib().lesgpu_get_scalar_staging(self._h))

    def get_tiles(self):
        t = np.zeros(5, dtype=np.int32)
        self._check(lib().lesgpu_get_tiles(self._h, t.ctypes.data), "get_tiles")
        return t.tolist()

    KERNEL_CLASSES = ["sem", "filter_props", "strain", "rhs_flow", "bc", "rhs_scalar"]

    def kernel_timing(self, on: bool = True):
        self._check(lib().lesgpu_kernel_timing(self._h, 1 if on else 0), "kernel_timing")

    def kernel_times(self) -> Dict[str, tuple]:
        nk = len(self.KERNEL_CLASSES)
        ms = np.zeros(nk)
        cnt = np.zeros(nk, dtype=np.int64)
        self._check(lib().lesgpu_kernel_times(self._h, ms.ctypes.data, cnt.ctypes.data, nk), "kernel_times")
        return {k: (float(ms[q]), int(cnt[q])) for q, k in enumerate(self.KERNEL_CLASSES)}

    @property
    def device_bytes(self) -> int:
        return lib().lesgpu_device_bytes(self._h)


class Solver:
    """``les_solver``: the reference's time loop with the step body on the GPU."""

    def __init__(self, cfg: SolverConfig, precision: int = FP64, start_step: int = 0, chem: str = CHEM_BIN,
                 tran: str = TRAN_BIN, device: int = 0):
        self.cfg = cfg
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self._c = LesgpuConfig.from_config(cfg, precision, device)
        h = C.c_void_p()
        rc = lib().les_solver_create(C.byref(self._c), chem.encode(), tran.encode(), start_step, C.byref(h))
        if rc != 0:
            raise LesgpuError(rc, "les_solver_create failed")
        self._h = h
        self.ctx = Context.__new__(Context)
        self.ctx.cfg = cfg
        self.ctx.shape = self.shape
        self.ctx._h = C.c_void_p(lib().les_solver_ctx(h))

    @classmethod
    def wrap(cls, handle, cfg: SolverConfig) -> "Solver":
        """A view of a les_solver owned elsewhere (an ensemble member); close() only detaches."""
        s = cls.__new__(cls)
        s.cfg = cfg
        s.shape = (cfg.nx, cfg.ny, cfg.nz)
        s._h = C.c_void_p(handle)
        s._owned = False
        s.ctx = Context.__new__(Context)
        s.ctx.cfg = cfg
        s.ctx.shape = s.shape
        s.ctx._h = C.c_void_p(lib().les_solver_ctx(s._h))
        return s

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise LesgpuError(rc, f"{what}: {lib().les_solver_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self.ctx._h = None
            if getattr(self, "_owned", True):
                lib().les_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_outputs(self, directory: Optional[str], flags: int):
        self._check(lib().les_solver_set_outputs(self._h, directory.encode() if directory else None, flags),
                    "set_outputs")

    def step(self, n: int = 1):
        for _ in range(n):
            self._check(lib().les_solver_step(self._h), "step")

    def run(self, n: int):
        self._check(lib().les_solver_run(self._h, n), "run")

    def run_device(self, n: int, chunk: int = 64):
        """n steps with the host side on the GPU (graph-replayed, no per-step round trip)."""
        self._check(lib().les_solver_run_device(self._h, n, chunk), "run_device")

    def loop_begin(self, chunk: int = 64):
        self._check(lib().les_solver_loop_begin(self._h, chunk), "loop_begin")

    def finish(self, directory: str, mode: int = 0):
        """End-of-run writes (checkpoint.bin, restart_info.txt, ...); mode RESUME_REFERENCE
        saves step 0 as the reference does, RESUME_FIXED the step reached plus les_resume.bin."""
        self._check(lib().les_solver_finish(self._h, directory.encode(), mode), "finish")

    def resume(self, directory: str, mode: int = 0) -> int:
        """The reference's auto-resume from `directory` (RESUME_REFERENCE keeps its defects,
        RESUME_FIXED continues the run exactly); returns the step the run continues from."""
        t = C.c_int(0)
        self._check(lib().les_solver_resume(self._h, directory.encode(), mode, C.byref(t)), "resume")
        return t.value

    def pstat_begin(self, edges: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """Accumulate the probe-row statistics on the device during device-loop runs; returns
        the edges in use (stats.default_edges when none are given)."""
        from . import stats
        e = edges or stats.default_edges(self.cfg.ly, self.cfg.inlet_velocity)
        a = {k: np.ascontiguousarray(e[k], dtype=np.float64) for k in ("y_mm", "g_rc", "g_ho", "u", "v")}
        assert len(a["u"]) == len(a["v"])
        self._check(lib().les_solver_pstat_begin(self._h, a["y_mm"].ctypes.data, len(a["y_mm"]) - 1,
                                                 a["g_rc"].ctypes.data, len(a["g_rc"]) - 1, a["g_ho"].ctypes.data,
                                                 len(a["g_ho"]) - 1, a["u"].ctypes.data, a["v"].ctypes.data,
                                                 len(a["u"]) - 1), "pstat_begin")
        self._pstat_edges = a
        return a

    def pstat_read(self) -> np.ndarray:
        out = np.empty(lib().les_solver_pstat_size(self._h))
        self._check(lib().les_solver_pstat_read(self._h, out.ctypes.data), "pstat_read")
        return out

    def profile_stats(self) -> Dict:
        """The device-accumulated statistics (stats.from_moments of pstat_read)."""
        from . import stats
        return stats.from_moments(self.pstat_read(), self._pstat_edges)

    def set_averaging(self, start_step: int):
        """Sum the time averages from t_loop >= start_step on (< 0: off)."""
        self._check(lib().les_solver_set_averaging(self._h, start_step), "set_averaging")

    def save_stats(self, path: str):
        self._check(lib().les_solver_save_stats(self._h, path.encode()), "save_stats")

    def load_stats(self, path: str):
        self._check(lib().les_solver_load_stats(self._h, path.encode()), "load_stats")

    def average_sums(self):
        """The ten running sums (AVG_NAMES) and the number of steps summed."""
        out = {k: np.empty(self.shape) for k in AVG_NAMES}
        ptrs = (C.c_void_p * 10)(*[out[k].ctypes.data for k in AVG_NAMES])
        n = C.c_int(0)
        rc = lib().lesgpu_avg_download(self.ctx._h, ptrs, C.byref(n))
        if rc:
            raise LesgpuError(rc, "lesgpu_avg_download failed")
        return out, n.value

    def reynolds_stresses(self):
        out = {k: np.empty(self.shape) for k in STRESS_NAMES}
        ptrs = (C.c_void_p * 7)(*[out[k].ctypes.data for k in STRESS_NAMES])
        n = C.c_int(0)
        self._check(lib().les_solver_reynolds_stresses(self._h, ptrs, C.byref(n)), "reynolds_stresses")
        return out, n.value

    def flush(self):
        self._check(lib().les_solver_flush(self._h), "flush")

    def loop_run(self, n: int):
        self._check(lib().les_solver_loop_run(self._h, n), "loop_run")

    def loop_end(self):
        self._check(lib().les_solver_loop_end(self._h), "loop_end")

    @property
    def t_loop(self) -> int:
        return lib().les_solver_t_loop(self._h)

    @property
    def last_dt(self) -> float:
        return lib().les_solver_last_dt(self._h)

    @property
    def rng_draws(self) -> int:
        return lib().les_solver_rng_draws(self._h)

    def vortices(self) -> np.ndarray:
        out = np.empty((self.cfg.num_vortices, 7), dtype=np.float64)
        lib().les_solver_vortices(self._h, out.ctypes.data)
        return out

    def attribute(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.int32)
        self._check(lib().les_solver_attribute(self._h, out.ctypes.data), "attribute")
        return out

    def state(self) -> Dict[str, np.ndarray]:
        return self.ctx.download_state()

    def field(self, name: str) -> np.ndarray:
        return self.ctx.field(name)

    def save_checkpoint(self, path: str, t: int):
        self._check(lib().les_solver_save_checkpoint(self._h, path.encode(), t), "save_checkpoint")

    def load_checkpoint(self, path: str) -> int:
        t = C.c_int()
        self._check(lib().les_solver_load_checkpoint(self._h, path.encode(), C.byref(t)), "load_checkpoint")
        return t.value
