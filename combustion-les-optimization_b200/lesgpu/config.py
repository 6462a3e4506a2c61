"""Run-time configuration of the solver step.

In the reference every item below is a compile-time ``#define`` (``les_combustion_solver.c``
lines 46-83, 136-262) or a function-local constant (``:2701-2703``, ``:2834``,
``:4101``).  Here they are one plain record, so grid size and model constants change
without recompiling, and an ensemble can give every member its own model constants.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from typing import Dict


@dataclass
class SolverConfig:
    # grid and box (les_combustion_solver.c:46-51)
    nx: int = 60
    ny: int = 20
    nz: int = 40
    lx: float = 0.12
    ly: float = 0.04
    lz: float = 0.08
    # inlet and SEM (:54-63)
    inlet_radius: float = 0.013
    rim_outer_radius: float = 0.005
    inlet_velocity: float = 4.0
    inlet_temperature: float = 300.0
    ambient_temperature: float = 300.0
    turbulence_intensity: float = 0.20
    num_vortices: int = 2000
    length_scale: float = 0.2 * 0.013
    # combustion (:66-70)
    s_l: float = 0.4
    initial_flame_front_i: int = 100
    burnt_gas_temperature: float = 2200.0
    # LES / turbulence (:75-78)
    pr_t: float = 0.5
    sc_t: float = 0.8
    d3: float = 2.35
    # time step control (:82-83)
    courant: float = 0.1
    courant_diffusion: float = 0.1
    # model constants (:257-262) and the nudging coefficient (:2834)
    cs_unburned: float = 0.1374
    cs_burnt: float = 0.4223
    cs_flame_boost: float = 0.2371
    accel_strength: float = 2.0361
    accel_width: float = 0.1126
    accel_center: float = 0.6697
    relax: float = 5000.0
    # SSR-SGS inputs (:154, :2701-2702)
    nu_unburnt: float = 1.5e-5
    rho_unburnt_approx: float = 1.2
    rho_burnt_approx: float = 0.2
    # mixture (:4101)
    equivalence_ratio: float = 1.1
    # misc switches
    weno_transition_step: int = 500          # :2740
    flame_accel: int = 1                     # USE_FLAME_ACCEL_MODEL, :208
    seed: int = 1234                         # srand() seed (the reference uses time(NULL))

    def as_dict(self) -> Dict:
        return dataclasses.asdict(self)

    def replace(self, **kw) -> "SolverConfig":
        return dataclasses.replace(self, **kw)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def _case(nx, ny, nz, lx, ly, lz, nv, i_f, u_in=5.0, ti=0.10, ell=0.004, courant=0.3, **kw):
    return SolverConfig(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, lz=lz, inlet_velocity=u_in,
                        turbulence_intensity=ti, num_vortices=nv, length_scale=ell,
                        initial_flame_front_i=i_f, courant=courant, **kw)


# Named cases.  "c1" .. "c3" are the 64x32x32 / 256x128x128 / 512x256x256 cases over a
# 0.128 x 0.064 x 0.064 m box with the flame plane at x = 0.03 m; "tiny"/"small" are
# the fixture grids at the same 2 mm spacing; "e128"/"e96" are the two ensemble grids.
PRESETS: Dict[str, SolverConfig] = {
    "tiny": _case(24, 12, 16, 0.048, 0.024, 0.032, nv=50, i_f=6),
    "small": _case(40, 16, 24, 0.080, 0.032, 0.048, nv=120, i_f=10),
    "c1": _case(64, 32, 32, 0.128, 0.064, 0.064, nv=200, i_f=15),
    "c2": _case(256, 128, 128, 0.128, 0.064, 0.064, nv=800, i_f=60),
    "c3": _case(512, 256, 256, 0.128, 0.064, 0.064, nv=3000, i_f=120, ti=0.15),
    "e128": _case(128, 64, 64, 0.128, 0.064, 0.064, nv=400, i_f=30),
    "e96": _case(96, 48, 48, 0.128, 0.064, 0.064, nv=300, i_f=22),
    "s192": _case(192, 96, 96, 0.128, 0.064, 0.064, nv=600, i_f=45),
    "reference_default": SolverConfig(),
}


def preset(name: str, **overrides) -> SolverConfig:
    return PRESETS[name].replace(**overrides)
