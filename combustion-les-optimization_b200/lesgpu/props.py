"""Species property files in the solver's Fortran-record format.

The solver reads two binary files at start-up (``les_combustion_solver.c:311-382``,
``load_chem_bin`` / ``load_tran_bin``), written upstream by ``generate_bins.py:114-177``
from Cantera/GRI data:

* ``chem.bin`` -- record 2 holds (MM, KK) at byte offsets 12/16; record 4 holds, per
  species, name[16], composition int[MM], 2 ints, MW (g/mol), 1 int, 3 doubles (the
  third is T_mid), NASA-7 high[7], NASA-7 low[7], after an 8-byte tag.
* ``tran.bin`` -- records 5/6/7 hold the conductivity fits (KK x 4), viscosity fits
  (KK x 4) and binary-diffusion fits (KK x KK x 4), each ``ln(prop) = a0 + a1 lnT +
  a2 ln^2T + a3 ln^3T`` in CGS units.

Cantera and the mechanism file are not available here, so :func:`synthetic_species`
provides a PLACEHOLDER property set with plausible magnitudes (cp/R from smooth
polynomials, mu/lambda/D as near-power laws anchored at 300 K).  These are not
GRI-Mech values; they only need to be fixed and shared so that every implementation of
the solver step sees the same inputs.  Slot 0 is propane (the solver's C3H8_INDEX).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from typing import List

NUM_SPECIES = 5
SPECIES_NAMES = ["C3H8", "O2", "N2", "CO2", "H2O"]
# element order used for the composition block of chem.bin
ELEMENTS = ["C", "H", "N", "O"]
_COMPOSITION = {
    "C3H8": [3, 8, 0, 0],
    "O2": [0, 0, 0, 2],
    "N2": [0, 0, 2, 0],
    "CO2": [1, 0, 0, 2],
    "H2O": [0, 2, 0, 1],
}
_ATOMIC_WEIGHT = {"C": 12.011, "H": 1.008, "N": 14.007, "O": 15.999}


@dataclass
class SpeciesSet:
    """Five species' data exactly as the solver's ``SpeciesData`` holds it
    (``les_combustion_solver.c:292-305``)."""

    names: List[str]
    mw: List[float]                      # g/mol
    t_mid: List[float]                   # K
    nasa_high: List[List[float]]         # [5][7]
    nasa_low: List[List[float]]          # [5][7]
    lam: List[List[float]]               # [5][4]  conductivity fit (erg/cm/s/K)
    eta: List[List[float]]               # [5][4]  viscosity fit (poise)
    dcoef: List[List[List[float]]] = field(default_factory=list)  # [5][5][4] (cm^2/s)


def _mw(name: str) -> float:
    comp = _COMPOSITION[name]
    return sum(n * _ATOMIC_WEIGHT[e] for n, e in zip(comp, ELEMENTS))


def _powerlaw_fit(value_300: float, expo: float, curv2: float, curv3: float) -> List[float]:
    """Coefficients of ln(prop) = a0 + a1 L + a2 L^2 + a3 L^3 (L = ln T) that pass
    through ``value_300`` at 300 K with local slope ``expo``."""
    L = math.log(300.0)
    a1 = expo - 2.0 * curv2 * L - 3.0 * curv3 * L * L
    a0 = math.log(value_300) - a1 * L - curv2 * L * L - curv3 * L * L * L
    return [a0, a1, curv2, curv3]


def _nasa_pair(c300: float, c1000: float, c3000: float) -> tuple:
    """Placeholder NASA-7 low/high cp/R polynomials: quadratic through the three anchor
    values, continuous at T_mid = 1000 K, plus small cubic/quartic terms so every
    power of T in the polynomial is exercised."""
    # low branch: a0 + a1 T + a2 T^2 through (300, c300), (1000, c1000) with a2 fixed
    a2 = -2.0e-7 * (c1000 - c300)
    a1 = ((c1000 - c300) - a2 * (1000.0 ** 2 - 300.0 ** 2)) / 700.0
    a0 = c300 - a1 * 300.0 - a2 * 300.0 ** 2
    low = [a0, a1, a2, 3.0e-11 * (c1000 - c300) / 10.0, -4.0e-15 * (c1000 - c300) / 10.0,
           -1000.0, 5.0]
    # subtract the small cubic/quartic contribution at 1000 K from a0 to stay continuous
    low[0] -= low[3] * 1000.0 ** 3 + low[4] * 1000.0 ** 4
    b2 = -1.0e-8 * (c3000 - c1000)
    b1 = ((c3000 - c1000) - b2 * (3000.0 ** 2 - 1000.0 ** 2)) / 2000.0
    b0 = c1000 - b1 * 1000.0 - b2 * 1000.0 ** 2
    high = [b0, b1, b2, 2.0e-13 * (c3000 - c1000), -1.0e-17 * (c3000 - c1000), -900.0, 4.0]
    high[0] -= high[3] * 1000.0 ** 3 + high[4] * 1000.0 ** 4
    return high, low


def synthetic_species() -> SpeciesSet:
    """The fixed placeholder property set used by every solver in this repository."""
    # cp/R anchors at 300 / 1000 / 3000 K
    cp_anchor = {
        "C3H8": (8.9, 20.0, 29.0),
        "O2": (3.55, 4.25, 4.65),
        "N2": (3.50, 3.90, 4.40),
        "CO2": (4.50, 6.60, 7.50),
        "H2O": (4.03, 4.95, 6.40),
    }
    mu300 = {"C3H8": 8.2e-6, "O2": 2.07e-5, "N2": 1.79e-5, "CO2": 1.50e-5, "H2O": 1.00e-5}
    lam300 = {"C3H8": 0.0180, "O2": 0.0266, "N2": 0.0260, "CO2": 0.0166, "H2O": 0.0190}
    names = list(SPECIES_NAMES)
    mw = [_mw(n) for n in names]
    t_mid = [1000.0] * NUM_SPECIES
    nasa_high, nasa_low, lam, eta = [], [], [], []
    for n in names:
        hi, lo = _nasa_pair(*cp_anchor[n])
        nasa_high.append(hi)
        nasa_low.append(lo)
        # CGS: poise = 10 Pa s; erg/(cm s K) = 1e5 W/(m K)
        eta.append(_powerlaw_fit(mu300[n] * 10.0, 0.70, 0.012, -0.0007))
        lam.append(_powerlaw_fit(lam300[n] * 1.0e5, 0.80, 0.015, -0.0009))
    dcoef = []
    for i in range(NUM_SPECIES):
        row = []
        for j in range(NUM_SPECIES):
            if i == j:
                row.append([0.0, 0.0, 0.0, 0.0])      # generate_bins.py writes zeros on the diagonal
            else:
                d300 = 0.16 * math.sqrt(56.0 / (mw[i] + mw[j]))   # cm^2/s
                row.append(_powerlaw_fit(d300, 1.75, 0.010, -0.0006))
        dcoef.append(row)
    return SpeciesSet(names, mw, t_mid, nasa_high, nasa_low, lam, eta, dcoef)


# --------------------------------------------------------------------------- file I/O

def _record(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def write_chem_bin(path: str, sp: SpeciesSet) -> None:
    """Write ``chem.bin`` in the record layout ``load_chem_bin`` reads
    (``les_combustion_solver.c:324-356``)."""
    mm, kk = len(ELEMENTS), NUM_SPECIES
    out = bytearray()
    out += _record(b"CHEM_SYNTHETIC\0\0".ljust(48, b"\0"))
    out += _record(struct.pack("<iii", 0, 0, 0) + struct.pack("<ii", mm, kk) + b"\0" * 60
                   + struct.pack("<d", 0.0))
    el = bytearray(b"ELEMENTS")
    for e in ELEMENTS:
        el += e.encode().ljust(16, b"\0") + struct.pack("<d", _ATOMIC_WEIGHT[e])
    out += _record(bytes(el))
    spr = bytearray(b"SPECIES ")
    for k in range(kk):
        spr += sp.names[k].encode().ljust(16, b"\0")
        spr += struct.pack(f"<{mm}i", *_COMPOSITION[sp.names[k]])
        spr += struct.pack("<ii", 0, 0)
        spr += struct.pack("<d", sp.mw[k])
        spr += struct.pack("<i", 0)
        spr += struct.pack("<ddd", 0.0, 0.0, sp.t_mid[k])
        spr += struct.pack("<7d", *sp.nasa_high[k])
        spr += struct.pack("<7d", *sp.nasa_low[k])
    out += _record(bytes(spr))
    out += _record(b"REACTION" + struct.pack("<iiddd", 1, 0, 0.0, 0.0, 0.0) + b"\0" * 48)
    with open(path, "wb") as f:
        f.write(bytes(out))


def write_tran_bin(path: str, sp: SpeciesSet) -> None:
    """Write ``tran.bin`` in the record layout ``load_tran_bin`` reads
    (``les_combustion_solver.c:359-382``)."""
    kk = NUM_SPECIES
    out = bytearray()
    out += _record(b"TRAN_SYNTHETIC\0\0".ljust(48, b"\0"))
    out += _record(struct.pack("<iiiii", 0, 0, 0, kk, 0))
    out += _record(b"PRESSURE" + struct.pack("<d", 101325.0))
    out += _record(b"".join(struct.pack("<d5di", 0.0, 0, 0, 0, 0, 0, 0) for _ in range(kk)))
    out += _record(b"".join(struct.pack("<4d", *sp.lam[k]) for k in range(kk)))
    out += _record(b"".join(struct.pack("<4d", *sp.eta[k]) for k in range(kk)))
    out += _record(b"".join(struct.pack("<4d", *sp.dcoef[i][j])
                            for i in range(kk) for j in range(kk)))
    with open(path, "wb") as f:
        f.write(bytes(out))


def _read_records(path: str) -> List[bytes]:
    recs = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos + 4 <= len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        if n < 0 or pos + 8 + n > len(data):
            raise ValueError(f"{path}: truncated Fortran record at byte {pos}")
        payload = data[pos + 4: pos + 4 + n]
        (n2,) = struct.unpack_from("<i", data, pos + 4 + n)
        if n2 != n:
            raise ValueError(f"{path}: record length mismatch ({n} vs {n2})")
        recs.append(payload)
        pos += 8 + n
    return recs


def read_species(chem_path: str, tran_path: str) -> SpeciesSet:
    """Read both files with the same offsets as ``load_chem_bin``/``load_tran_bin``."""
    rc = _read_records(chem_path)
    if len(rc) < 4:
        raise ValueError(f"{chem_path}: expected at least 4 records, found {len(rc)}")
    mm, kk = struct.unpack_from("<ii", rc[1], 12)
    if kk != NUM_SPECIES:
        raise ValueError(f"{chem_path}: solver needs {NUM_SPECIES} species, file has {kk}")
    per = 16 + 4 * mm + 8 + 8 + 4 + 24 + 2 * 56
    names, mw, t_mid, hi, lo = [], [], [], [], []
    for k in range(kk):
        base = 8 + k * per
        names.append(rc[3][base: base + 16].split(b"\0")[0].decode().strip())
        mwo = base + 16 + 4 * mm + 8
        mw.append(struct.unpack_from("<d", rc[3], mwo)[0])
        tmo = mwo + 8 + 4 + 16
        t_mid.append(struct.unpack_from("<d", rc[3], tmo)[0])
        hi.append(list(struct.unpack_from("<7d", rc[3], tmo + 8)))
        lo.append(list(struct.unpack_from("<7d", rc[3], tmo + 8 + 56)))
    rt = _read_records(tran_path)
    if len(rt) < 7:
        raise ValueError(f"{tran_path}: expected at least 7 records, found {len(rt)}")
    lam = [list(struct.unpack_from("<4d", rt[4], 32 * k)) for k in range(kk)]
    eta = [list(struct.unpack_from("<4d", rt[5], 32 * k)) for k in range(kk)]
    dco = [[list(struct.unpack_from("<4d", rt[6], 32 * (i * kk + j))) for j in range(kk)]
           for i in range(kk)]
    return SpeciesSet(names, mw, t_mid, hi, lo, lam, eta, dco)
