#!/usr/bin/env python3
"""Build the REFERENCE solver itself as an oracle (test infrastructure only).

This recipe compiles ``les_combustion_solver.c`` from the reference tree into
``oracle/_ref/<config>/les_ref`` after a textual patch of its compile-time macros:

* grid and box (``NX NY NZ LX LY LZ``, ``les_combustion_solver.c:46-51``),
* inlet / SEM macros (``INLET_VELOCITY``, ``INLET_TURBULENCE_INTENSITY``,
  ``NUM_VORTICES``, ``TURBULENT_LENGTH_SCALE``, ``:56-63``),
* ``INITIAL_FLAME_FRONT_I`` (``:69``) and ``COURANT_NUMBER`` (``:82``),
* ``OUTPUT_DIR`` -> ``"./"`` (``:93``),
* the six model constants (``:257-262``) and the local ``RELAXATION_COEFF`` (``:2834``)
  become globals read from the environment (defaults are the reference values),
* ``srand(time(NULL))`` -> ``srand(seed)`` (``:4085``), ``start_step`` and
  ``total_steps`` (``:4139``, ``:4377``) from the environment,
* a hook after ``apply_boundary_conditions`` (``:4555``) that dumps the state in the
  ``checkpoint.bin`` field order plus ``nu_t``/``S_mag`` and prints the per-step wall
  time (``omp_get_wtime``), and a hook after the stage-1 ``calculate_RHS`` (``:4429``)
  that dumps the RHS intermediates for per-kernel checks,
* ``output_vtk`` returns immediately when ``LES_REF_NOVTK`` is set (timing runs),
* the inflow loop of ``apply_boundary_conditions`` (``:2978``), which draws three
  ``rand()`` values per inlet cell inside ``#pragma omp parallel for``, runs on one thread
  when ``LES_REF_SERIAL_BC=1``: the draws then come in the serial (j, k) order whatever
  ``OMP_NUM_THREADS`` is, so a multi-threaded run is comparable with the GPU solver (with
  several threads the draw order depends on the OpenMP schedule and glibc's lock).  Every
  other loop keeps its threads; only the order of the OpenMP sums (``<rho_f>``, ``:2538``)
  still depends on the thread count, at rounding level,
* with ``LES_REF_DUMP_FIRST=1`` the state after the first step is dumped as well as every
  ``LES_REF_DUMP_EVERY``-th.

Nothing else in the solver is touched.  The reference tree is only read; all outputs go
under ``oracle/_ref/``.  The reference checkout is ``$LES_REFERENCE_DIR``, else a
``reference`` directory beside this repository.  Usage::

    python oracle/build_ref.py [--ref /path/to/reference] [--config NAME ...]
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_ROOT = os.path.join(HERE, "_ref")


def default_ref() -> str:
    """The reference checkout: ``$LES_REFERENCE_DIR``, else ``../reference`` beside the repository."""
    env = os.environ.get("LES_REFERENCE_DIR")
    if env:
        return env
    return os.path.normpath(os.path.join(os.path.dirname(HERE), "..", "reference"))


def ref_present(ref_dir: str = None) -> bool:
    return os.path.exists(os.path.join(ref_dir or default_ref(), "les_combustion_solver.c"))


# Grid configurations that the oracle binary is compiled for.  Grid sizes and the SEM
# vortex count are array dimensions in the reference, so each needs its own binary.
CONFIGS = {
    # small grids for golden fixtures and fast parity checks (dx = dy = dz = 2 mm)
    "tiny": dict(nx=24, ny=12, nz=16, lx=0.048, ly=0.024, lz=0.032, u_in=5.0, ti=0.10,
                 nv=50, ell=0.004, i_f=6, courant=0.3),
    "small": dict(nx=40, ny=16, nz=24, lx=0.080, ly=0.032, lz=0.048, u_in=5.0, ti=0.10,
                  nv=120, ell=0.004, i_f=10, courant=0.3),
    # 64x32x32 over 0.128 x 0.064 x 0.064 m, 200 eddies of 4 mm, front at x = 0.03 m
    "c1": dict(nx=64, ny=32, nz=32, lx=0.128, ly=0.064, lz=0.064, u_in=5.0, ti=0.10,
               nv=200, ell=0.004, i_f=15, courant=0.3),
    # 256x128x128 over the same box, 800 eddies, front at x = 0.03 m (i = 60)
    "c2": dict(nx=256, ny=128, nz=128, lx=0.128, ly=0.064, lz=0.064, u_in=5.0, ti=0.10,
               nv=800, ell=0.004, i_f=60, courant=0.3),
    # the two batched-ensemble grids
    "e128": dict(nx=128, ny=64, nz=64, lx=0.128, ly=0.064, lz=0.064, u_in=5.0, ti=0.10,
                 nv=400, ell=0.004, i_f=30, courant=0.3),
    "e96": dict(nx=96, ny=48, nz=48, lx=0.128, ly=0.064, lz=0.064, u_in=5.0, ti=0.10,
                nv=300, ell=0.004, i_f=22, courant=0.3),
}

HOOKS = r'''
/* ---- oracle hooks (added by oracle/build_ref.py; not part of the reference) ---- */
double les_ref_cs_unburned = 0.1374, les_ref_cs_burnt = 0.4223, les_ref_cs_boost = 0.2371;
double les_ref_accel_strength = 2.0361, les_ref_accel_width = 0.1126, les_ref_accel_center = 0.6697;
double les_ref_relax = 5000.0;
unsigned int les_ref_seed = 1234u;
int les_ref_start = 0, les_ref_steps = 10, les_ref_dump_every = 0, les_ref_novtk = 0, les_ref_rhs_dump_step = -1;
int les_ref_serial_bc = 0, les_ref_dump_first = 0;
double les_ref_t0 = 0.0, les_ref_tprev = 0.0;
static double les_ref_envd(const char* n, double d) { const char* s = getenv(n); return s ? strtod(s, NULL) : d; }
static int les_ref_envi(const char* n, int d) { const char* s = getenv(n); return s ? atoi(s) : d; }
void les_ref_init(void) {
    les_ref_cs_unburned = les_ref_envd("LES_REF_CS_UNBURNED", les_ref_cs_unburned);
    les_ref_cs_burnt = les_ref_envd("LES_REF_CS_BURNT", les_ref_cs_burnt);
    les_ref_cs_boost = les_ref_envd("LES_REF_CS_BOOST", les_ref_cs_boost);
    les_ref_accel_strength = les_ref_envd("LES_REF_ACCEL_STRENGTH", les_ref_accel_strength);
    les_ref_accel_width = les_ref_envd("LES_REF_ACCEL_WIDTH", les_ref_accel_width);
    les_ref_accel_center = les_ref_envd("LES_REF_ACCEL_CENTER", les_ref_accel_center);
    les_ref_relax = les_ref_envd("LES_REF_RELAX", les_ref_relax);
    les_ref_seed = (unsigned int)les_ref_envi("LES_REF_SEED", 1234);
    les_ref_start = les_ref_envi("LES_REF_START", 0);
    les_ref_steps = les_ref_envi("LES_REF_STEPS", 10);
    les_ref_dump_every = les_ref_envi("LES_REF_DUMP_EVERY", 0);
    les_ref_novtk = les_ref_envi("LES_REF_NOVTK", 0);
    les_ref_rhs_dump_step = les_ref_envi("LES_REF_RHS_DUMP_STEP", -1);
    les_ref_serial_bc = les_ref_envi("LES_REF_SERIAL_BC", 0);
    les_ref_dump_first = les_ref_envi("LES_REF_DUMP_FIRST", 0);
}
'''

MAIN_HOOKS = r'''
static void les_ref_put(FILE* f, Grid3D a) { fwrite(a, sizeof(double), (size_t)NX * NY * NZ, f); }
void les_ref_after_step(int t, double dt) {
    double now = omp_get_wtime();
    fprintf(stderr, "LESREF_STEP %d %.17g %.9f\n", t, dt, now - les_ref_tprev);
    les_ref_tprev = now;
    int n = t + 1 - les_ref_start;
    if ((les_ref_dump_every > 0 && n % les_ref_dump_every == 0) || (les_ref_dump_first && n == 1)) {
        char p[64]; sprintf(p, "state_%06d.bin", n);
        FILE* f = fopen(p, "wb");
        if (!f) return;
        fwrite(&t, sizeof(int), 1, f); fwrite(&dt, sizeof(double), 1, f);
        les_ref_put(f, u); les_ref_put(f, v); les_ref_put(f, w); les_ref_put(f, T);
        les_ref_put(f, G); les_ref_put(f, rho);
        for (int sp = 0; sp < NUM_SPECIES; sp++) les_ref_put(f, Yk[sp]);
        les_ref_put(f, nu_t); les_ref_put(f, S_mag);
        fclose(f);
    }
}
void les_ref_after_rhs1(int t) {
    if (t != les_ref_rhs_dump_step) return;
    FILE* f = fopen("rhs1.bin", "wb");
    if (!f) return;
    les_ref_put(f, u_filtered); les_ref_put(f, v_filtered); les_ref_put(f, w_filtered);
    les_ref_put(f, T_filtered); les_ref_put(f, G_filtered); les_ref_put(f, rho_filtered);
    for (int sp = 0; sp < NUM_SPECIES; sp++) les_ref_put(f, Yk_filtered[sp]);
    les_ref_put(f, nu); les_ref_put(f, mu_mix); les_ref_put(f, nu_t); les_ref_put(f, S_mag);
    les_ref_put(f, ST_turbulent); les_ref_put(f, Cp_mix); les_ref_put(f, lambda_mix); les_ref_put(f, alpha);
    for (int sp = 0; sp < NUM_SPECIES; sp++) les_ref_put(f, Dk[sp]);
    les_ref_put(f, k1_rhou); les_ref_put(f, k1_rhov); les_ref_put(f, k1_rhow);
    les_ref_put(f, k1_T); les_ref_put(f, k1_G);
    for (int sp = 0; sp < NUM_SPECIES; sp++) les_ref_put(f, k1_Yk[sp]);
    fclose(f);
}
'''

# Order of the fields in state_*.bin after the (int t, double dt) header.
STATE_FIELDS = ["u", "v", "w", "T", "G", "rho", "Y0", "Y1", "Y2", "Y3", "Y4", "nu_t", "S_mag"]
# Order of the fields in rhs1.bin.
RHS1_FIELDS = (["u_f", "v_f", "w_f", "T_f", "G_f", "rho_f"] + [f"Y{k}_f" for k in range(5)]
               + ["nu", "mu_mix", "nu_t", "S_mag", "ST", "Cp", "lambda", "alpha"]
               + [f"D{k}" for k in range(5)]
               + ["k_rhou", "k_rhov", "k_rhow", "k_T", "k_G"] + [f"k_Y{k}" for k in range(5)])


def _sub(src: str, pattern: str, repl: str, flags: int = re.M) -> str:
    new, n = re.subn(pattern, lambda _m: repl, src, flags=flags)
    if n != 1:
        raise RuntimeError(f"patch {pattern!r} matched {n} times (expected exactly 1)")
    return new


def patch_source(src: str, cfg: dict) -> str:
    s = src
    for name, key in (("NX", "nx"), ("NY", "ny"), ("NZ", "nz")):
        s = _sub(s, rf"^#define {name} \d+\b.*$", f"#define {name} {cfg[key]}")
    for name, key in (("LX", "lx"), ("LY", "ly"), ("LZ", "lz")):
        s = _sub(s, rf"^#define {name} [0-9.]+\s*$", f"#define {name} {cfg[key]!r}")
    s = _sub(s, r"^#define INLET_VELOCITY 4\.0\b.*$", f"#define INLET_VELOCITY {cfg['u_in']!r}")
    s = _sub(s, r"^#define INLET_TURBULENCE_INTENSITY 0\.20\b.*$",
             f"#define INLET_TURBULENCE_INTENSITY {cfg['ti']!r}")
    s = _sub(s, r"^#define NUM_VORTICES 2000\b.*$", f"#define NUM_VORTICES {cfg['nv']}")
    s = _sub(s, r"^#define TURBULENT_LENGTH_SCALE \(0\.2 \* INLET_RADIUS\).*$",
             f"#define TURBULENT_LENGTH_SCALE ({cfg['ell']!r})")
    s = _sub(s, r"^#define INITIAL_FLAME_FRONT_I 100\b.*$",
             f"#define INITIAL_FLAME_FRONT_I {cfg['i_f']}")
    s = _sub(s, r"^#define COURANT_NUMBER 0\.1\b.*$", f"#define COURANT_NUMBER {cfg['courant']!r}")
    s = _sub(s, r'^#define OUTPUT_DIR "D:.*$', '#define OUTPUT_DIR "./"')
    for macro, var in (("FLAME_ACCEL_STRENGTH", "les_ref_accel_strength"),
                       ("FLAME_ACCEL_WIDTH", "les_ref_accel_width"),
                       ("FLAME_ACCEL_CENTER", "les_ref_accel_center"),
                       ("CS_UNBURNED", "les_ref_cs_unburned"),
                       ("CS_BURNT", "les_ref_cs_burnt"),
                       ("CS_FLAME_BOOST", "les_ref_cs_boost")):
        s = _sub(s, rf"^#define {macro}\s+[0-9.]+\s*$", f"#define {macro} {var}")
    s = _sub(s, r"const double RELAXATION_COEFF = 5000\.0;", "const double RELAXATION_COEFF = les_ref_relax;")
    s = _sub(s, r"^#include <signal\.h>\s*$", "#include <signal.h>\n" + HOOKS)
    s = _sub(s, r"srand\(time\(NULL\)\);", "les_ref_init(); srand(les_ref_seed);")
    s = _sub(s, r"int start_step = 0;", "int start_step = les_ref_start;")
    s = _sub(s, r"int total_steps = \(int\)\(SIMULATION_TIME / DT_sim\);",
             "int total_steps = les_ref_start + les_ref_steps;")
    s = _sub(s, r'printf\("\\n--- Simulation Loop Start ---\\n"\);',
             'printf("\\n--- Simulation Loop Start ---\\n"); les_ref_t0 = les_ref_tprev = omp_get_wtime();')
    s = _sub(s, r"^(\s*)apply_boundary_conditions\(attribute, u, v, w, rhou, rhov, rhow, G, T, P, Yk, rho\);",
             "        apply_boundary_conditions(attribute, u, v, w, rhou, rhov, rhow, G, T, P, Yk, rho);"
             " les_ref_after_step(t_loop, DT_sim);")
    s = _sub(s, r"calculate_RHS\(t_loop, u, v, w, T, G, Yk, rho, k1_rhou, k1_rhov, k1_rhow, k1_T, k1_G, k1_Yk\);",
             "calculate_RHS(t_loop, u, v, w, T, G, Yk, rho, k1_rhou, k1_rhov, k1_rhow, k1_T, k1_G, k1_Yk);"
             " les_ref_after_rhs1(t_loop);")
    s = _sub(s, r"^void output_vtk\(int t\) \{", "void output_vtk(int t) { if (les_ref_novtk) return;")
    s, n = re.subn(r"(\(i=0, i=NX-1\) ---[^\n]*\n[^\n]*\n[ \t]*)#pragma omp parallel for(\r?\n)",
                   lambda m: m.group(1) + "#pragma omp parallel for if(!les_ref_serial_bc)" + m.group(2), s)
    if n != 1:
        raise RuntimeError(f"inflow-loop pragma patch matched {n} times (expected exactly 1)")
    s = _sub(s, r"^int main\(int argc, char \*argv\[\]\) \{", MAIN_HOOKS + "\nint main(int argc, char *argv[]) {")
    return s


def build(ref_dir: str, names, quiet: bool = False) -> None:
    src_path = os.path.join(ref_dir, "les_combustion_solver.c")
    if not os.path.exists(src_path):
        raise FileNotFoundError(f"reference source not found: {src_path}")
    with open(src_path, "r", encoding="utf-8") as f:
        src = f.read()
    data_dir = os.path.join(os.path.dirname(HERE), "combustion-les-optimization_b200", "data")
    for name in names:
        cfg = CONFIGS[name]
        out = os.path.join(OUT_ROOT, name)
        os.makedirs(out, exist_ok=True)
        csrc = os.path.join(out, "les_ref.c")
        with open(csrc, "w", encoding="utf-8") as f:
            f.write(patch_source(src, cfg))
        for fn in ("chem.bin", "tran.bin"):
            shutil.copyfile(os.path.join(data_dir, fn), os.path.join(out, fn))
        exe = os.path.join(out, "les_ref")
        # -ffp-contract=off: the reference is built for baseline x86-64 (no FMA), and the
        # oracle keeps that arithmetic even if the host compiler targets FMA hardware.
        cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-w", csrc, "-o", exe, "-lm"]
        subprocess.run(cmd, check=True)
        if not quiet:
            print(f"built {exe}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ref", default=default_ref())
    ap.add_argument("--config", action="append", choices=sorted(CONFIGS))
    args = ap.parse_args(argv)
    build(args.ref, args.config or sorted(CONFIGS))
    return 0


if __name__ == "__main__":
    sys.exit(main())
