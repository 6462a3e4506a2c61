"""Profile statistics of the probe rows (the solver's probe_data_flame_region_loc*.csv).

These are the quantities the reference's post-processing draws from the probe files and
that its Bayesian optimiser scores; they are the outputs whose error the FP32 precision
form states against the FP64 form:

* ``flame_profile``   -- analysis.py:112-154 (task_1_3_flame_profile): fluctuations about the
  global means, binned by distance from the flame front (0.5 mm bins from the smallest
  y_relative, right-closed as pandas.cut), per-bin means of u, v, w, G and of the Reynolds
  stresses u'u', v'v', w'w', u'v';
* ``stress_vs_g``     -- analysis.py:215-257 (task_1_6_reynolds_stress_vs_g_binned): G bins
  (0, 0.05], ..., (1.0, 1.05]; fluctuations about the per-bin means; per-bin means of
  u'u', v'v', u'v'; also the per-bin mean velocities;
* ``uv_vs_g``         -- bayesian_optimizer.py:71-117 (load_and_compute_reynolds_stress):
  num_bins half-open G bins [a, b) over [0, 1], <u'v'> = <uv> - <u><v> for bins with at
  least 10 rows, NaN otherwise;
* ``conditional_pdfs``-- analysis.py:82-110 (task_1_2_conditional_pdfs) draws kernel density
  estimates of u and v for unburnt (G < 0.5) and burnt (G >= 0.5) rows; here the same
  conditional samples are summarised as normalised histograms on fixed edges.

Rows are read from the CSV files (``read_probe_csv``) or built from the device loop's probe
history.  All statistics are computed in float64 with numpy.
"""
from __future__ import annotations

import io
import os
from typing import Dict, Optional

import numpy as np

COLUMNS = ["timestep", "x_location", "y_flame", "y_physical", "y_relative", "u", "v", "w", "G", "nu_t", "S_mag"]


def read_probe_csv(path: str) -> Dict[str, np.ndarray]:
    """One probe file as a dict of float64 columns (the header written by the solver)."""
    with open(path) as fp:
        header = fp.readline().strip().split(",")
    if header != COLUMNS:
        raise ValueError(f"{path}: unexpected header {header}")
    with open(path) as fp:
        fp.readline()
        body = fp.read()
    if not body.strip():
        return {c: np.zeros(0) for c in COLUMNS}
    data = np.loadtxt(io.StringIO(body), delimiter=",", ndmin=2)
    if data.size == 0:
        return {c: np.zeros(0) for c in COLUMNS}
    return {c: data[:, q].astype(np.float64) for q, c in enumerate(COLUMNS)}


def read_probe_dir(directory: str, loc: int) -> Dict[str, np.ndarray]:
    return read_probe_csv(os.path.join(directory, f"probe_data_flame_region_loc{loc}.csv"))


def _right_closed_bins(x: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """Bin index of each x for the intervals (e[b], e[b+1]] (pandas.cut default); -1 outside."""
    b = np.searchsorted(edges, x, side="left") - 1
    b[(x <= edges[0]) | (x > edges[-1])] = -1
    return b


def _group_means(b: np.ndarray, nb: int, cols: Dict[str, np.ndarray]):
    """Per-bin means of each column over the occupied bins (groupby(...).mean(), observed=True)."""
    ok = b >= 0
    cnt = np.bincount(b[ok], minlength=nb).astype(np.float64)
    occ = cnt > 0
    out = {}
    for k, v in cols.items():
        s = np.bincount(b[ok], weights=v[ok], minlength=nb)
        out[k] = s[occ] / cnt[occ]
    return occ, out


def flame_edges(rows: Dict[str, np.ndarray]) -> np.ndarray:
    """The 0.5 mm y_relative bin edges of analysis.py:126-127, from the rows' own range."""
    y_mm = rows["y_relative"] * 1000
    return np.arange(y_mm.min(), y_mm.max() + 0.5, 0.5)


def flame_profile(rows: Dict[str, np.ndarray], edges: Optional[np.ndarray] = None) -> Dict[str, np.ndarray]:
    """analysis.py:112-130: Reynolds stresses about the global means, binned in y_relative.
    ``edges`` (mm) replaces the rows' own bins, to compare two runs on the same bins."""
    u, v, w, G = rows["u"], rows["v"], rows["w"], rows["G"]
    if len(u) == 0:
        return {k: np.zeros(0) for k in ("bin_center", "u", "v", "w", "G", "re_uu", "re_vv", "re_ww", "re_uv")}
    up, vp, wp = u - u.mean(), v - v.mean(), w - w.mean()
    y_mm = rows["y_relative"] * 1000
    if edges is None:
        edges = flame_edges(rows)
    b = _right_closed_bins(y_mm, edges)
    occ, m = _group_means(b, len(edges) - 1, {"u": u, "v": v, "w": w, "G": G, "re_uu": up * up, "re_vv": vp * vp,
                                               "re_ww": wp * wp, "re_uv": up * vp})
    m["bin_center"] = (0.5 * (edges[:-1] + edges[1:]))[occ]
    return m


def stress_vs_g(rows: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """analysis.py:218-236: conditional Reynolds stresses in 0.05-wide G bins."""
    u, v, w, G = rows["u"], rows["v"], rows["w"], rows["G"]
    edges = np.arange(0.0, 1.05, 0.05)
    nb = len(edges) - 1
    b = _right_closed_bins(G, edges)
    ok = b >= 0
    cnt = np.bincount(b[ok], minlength=nb).astype(np.float64)
    occ = cnt > 0
    mean = {}
    for k, x in (("u", u), ("v", v), ("w", w)):
        s = np.bincount(b[ok], weights=x[ok], minlength=nb)
        mean[k] = np.divide(s, cnt, out=np.zeros(nb), where=cnt > 0)
    bb = b[ok]
    up = u[ok] - mean["u"][bb]
    vp = v[ok] - mean["v"][bb]
    out = {}
    for k, x in (("uu_cond", up * up), ("vv_cond", vp * vp), ("uv_cond", up * vp)):
        out[k] = (np.bincount(bb, weights=x, minlength=nb) / np.maximum(cnt, 1))[occ]
    for k in ("u", "v", "w"):
        out[f"{k}_mean"] = mean[k][occ]
    out["G_center"] = (0.5 * (edges[:-1] + edges[1:]))[occ]
    return out


def uv_vs_g(rows: Dict[str, np.ndarray], num_bins: int = 20):
    """bayesian_optimizer.py:98-117: <u'v'> per half-open G bin; NaN for bins with < 10 rows."""
    u, v, G = rows["u"], rows["v"], rows["G"]
    edges = np.linspace(0.0, 1.0, num_bins + 1)
    centers = 0.5 * (edges[:-1] + edges[1:])
    stress = np.full(num_bins, np.nan)
    for b in range(num_bins):
        m = (G >= edges[b]) & (G < edges[b + 1])
        if m.sum() < 10:
            continue
        stress[b] = (u[m] * v[m]).mean() - u[m].mean() * v[m].mean()
    return centers, stress


def conditional_pdfs(rows: Dict[str, np.ndarray], edges_u: np.ndarray, edges_v: np.ndarray):
    """Normalised histograms of u and v for unburnt (G < 0.5) and burnt (G >= 0.5) rows."""
    G = rows["G"]
    out = {}
    for tag, m in (("unburnt", G < 0.5), ("burnt", G >= 0.5)):
        for k, e in (("u", edges_u), ("v", edges_v)):
            x = rows[k][m]
            if len(x) == 0:
                out[f"{k}_{tag}"] = np.zeros(len(e) - 1)
            else:
                h, _ = np.histogram(x, bins=e, density=True)
                out[f"{k}_{tag}"] = h
    return out


def profile_error(a: np.ndarray, b: np.ndarray, ref_scale: Optional[float] = None) -> float:
    """Relative L2 difference ||a - b|| / ||b|| over the entries finite in both (NaN bins
    skipped); ``ref_scale`` replaces ||b|| for profiles that cross zero."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return float("inf")
    ok = np.isfinite(a) & np.isfinite(b)
    if not ok.any():
        return 0.0
    d = np.linalg.norm(a[ok] - b[ok])
    nb = ref_scale if ref_scale is not None else np.linalg.norm(b[ok])
    return float(d / nb) if nb > 0 else float(d)


def compare_profiles(rows_a: Dict[str, np.ndarray], rows_b: Dict[str, np.ndarray]) -> Dict[str, float]:
    """Per-profile relative L2 errors of run a against run b (b is the reference run)."""
    err = {}
    if len(rows_b["u"]) and len(rows_a["u"]):
        e = flame_edges(rows_b)
        fa, fb = flame_profile(rows_a, e), flame_profile(rows_b, e)
        common, ia, ib = np.intersect1d(fa["bin_center"], fb["bin_center"], return_indices=True)
        for k in ("u", "re_uu", "re_vv", "re_ww", "re_uv"):
            err[f"flame_profile.{'mean_u' if k == 'u' else k}"] = profile_error(fa[k][ia], fb[k][ib])
    sa, sb = stress_vs_g(rows_a), stress_vs_g(rows_b)
    if len(sa["G_center"]) == len(sb["G_center"]) and np.allclose(sa["G_center"], sb["G_center"]):
        for k in ("u_mean", "uu_cond", "vv_cond", "uv_cond"):
            err[f"stress_vs_G.{k}"] = profile_error(sa[k], sb[k])
    else:
        err["stress_vs_G.bins_differ"] = float("inf")
    _, ua = uv_vs_g(rows_a)
    _, ub = uv_vs_g(rows_b)
    err["uv_vs_G"] = profile_error(ua, ub)
    lo_u, hi_u = np.percentile(rows_b["u"], [0.5, 99.5]) if len(rows_b["u"]) else (0.0, 1.0)
    lo_v, hi_v = np.percentile(rows_b["v"], [0.5, 99.5]) if len(rows_b["v"]) else (0.0, 1.0)
    eu, ev = np.linspace(lo_u, hi_u, 41), np.linspace(lo_v, hi_v, 41)
    pa, pb = conditional_pdfs(rows_a, eu, ev), conditional_pdfs(rows_b, eu, ev)
    for k in pa:
        err[f"pdf.{k}"] = profile_error(pa[k], pb[k])
    return err
