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

``from_moments`` turns the moment sums that the solver accumulates on the device
(``lesgpu_pstat_*``, no probe files) into the same four statistics.
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


# ----------------------------------------------------------------- device moment sums

def default_edges(ly: float, inlet_velocity: float) -> Dict[str, np.ndarray]:
    """The bins les_solver_pstat_begin uses when given no edges (start + b * step)."""
    ly_mm = 1000.0 * ly
    ny_b = int(2.0 * ly_mm / 0.5 + 0.5)
    U = inlet_velocity
    e = {"y_mm": -ly_mm + np.arange(ny_b + 1) * 0.5,
         "g_rc": np.arange(21) * 0.05,
         "g_ho": np.append(np.arange(20) * (1.0 / 20), 1.0),
         "u": np.append(-U + np.arange(40) * (4.0 * U / 40), 3.0 * U),
         "v": np.append(-2.0 * U + np.arange(40) * (4.0 * U / 40), 2.0 * U)}
    return e


def moments_size(edges: Dict[str, np.ndarray]) -> int:
    ny, nrc, nho, npdf = (len(edges[k]) - 1 for k in ("y_mm", "g_rc", "g_ho", "u"))
    return 4 + 9 * ny + 7 * nrc + 4 * nho + 4 * npdf


def from_moments(sums: np.ndarray, edges: Dict[str, np.ndarray]) -> Dict[str, Dict]:
    """The statistics of ``flame_profile(rows, edges['y_mm'])``, ``stress_vs_g``, ``uv_vs_g``
    and ``conditional_pdfs(rows, edges['u'], edges['v'])`` from the device moment sums (layout
    of lesgpu_pstat_read).  Means of squared fluctuations come from the raw moments:
    <(x - m)^2> = <x^2> - 2 m <x> + m^2."""
    s = np.asarray(sums, dtype=np.float64)
    ny, nrc, nho, npdf = (len(edges[k]) - 1 for k in ("y_mm", "g_rc", "g_ho", "u"))
    if len(s) != moments_size(edges):
        raise ValueError("moment vector does not match the edges")
    N, su, sv, sw = s[0:4]
    out = {}
    # flame_profile: fluctuations about the global means
    Y = s[4:4 + 9 * ny].reshape(ny, 9)
    occ = Y[:, 0] > 0
    n = Y[occ, 0]
    mu, mv, mw = (su / N, sv / N, sw / N) if N > 0 else (0.0, 0.0, 0.0)
    fp = {"bin_center": (0.5 * (edges["y_mm"][:-1] + edges["y_mm"][1:]))[occ],
          "u": Y[occ, 1] / n, "v": Y[occ, 2] / n, "w": Y[occ, 3] / n, "G": Y[occ, 4] / n,
          "re_uu": (Y[occ, 5] - 2.0 * mu * Y[occ, 1]) / n + mu * mu,
          "re_vv": (Y[occ, 6] - 2.0 * mv * Y[occ, 2]) / n + mv * mv,
          "re_ww": (Y[occ, 7] - 2.0 * mw * Y[occ, 3]) / n + mw * mw,
          "re_uv": (Y[occ, 8] - mv * Y[occ, 1] - mu * Y[occ, 2]) / n + mu * mv}
    out["flame_profile"] = fp
    # stress_vs_g: fluctuations about the per-bin means
    o = 4 + 9 * ny
    Rc = s[o:o + 7 * nrc].reshape(nrc, 7)
    occ = Rc[:, 0] > 0
    n = Rc[occ, 0]
    bu, bv, bw = Rc[occ, 1] / n, Rc[occ, 2] / n, Rc[occ, 3] / n
    out["stress_vs_g"] = {"uu_cond": Rc[occ, 4] / n - bu * bu, "vv_cond": Rc[occ, 5] / n - bv * bv,
                          "uv_cond": Rc[occ, 6] / n - bu * bv, "u_mean": bu, "v_mean": bv, "w_mean": bw,
                          "G_center": (0.5 * (edges["g_rc"][:-1] + edges["g_rc"][1:]))[occ]}
    # uv_vs_g: bins with fewer than 10 rows are NaN
    o += 7 * nrc
    Ho = s[o:o + 4 * nho].reshape(nho, 4)
    stress = np.full(nho, np.nan)
    ok = Ho[:, 0] >= 10
    n = Ho[ok, 0]
    stress[ok] = Ho[ok, 3] / n - (Ho[ok, 1] / n) * (Ho[ok, 2] / n)
    out["uv_vs_g"] = (0.5 * (edges["g_ho"][:-1] + edges["g_ho"][1:]), stress)
    # conditional PDFs: density-normalised histograms
    o += 4 * nho
    H = s[o:o + 4 * npdf].reshape(4, npdf)
    pdfs = {}
    for q, (k, tag) in enumerate((("u", "unburnt"), ("v", "unburnt"), ("u", "burnt"), ("v", "burnt"))):
        c = H[q]
        w = np.diff(edges[k])
        tot = c.sum()
        pdfs[f"{k}_{tag}"] = c / (tot * w) if tot > 0 else np.zeros(npdf)
    out["conditional_pdfs"] = pdfs
    return out


def probe_rows(lines: np.ndarray, t0: int, dy: float, x_locations: np.ndarray) -> Dict[str, np.ndarray]:
    """Rows of record_flame_region_data (les_combustion_solver.c:3419-3466) at full precision,
    from probe lines shaped (steps, stations, NY, 6) = u, v, w, G, nu_t, S_mag."""
    cols = {c: [] for c in COLUMNS}
    steps, nst, ny, _ = lines.shape
    for q in range(steps):
        for n in range(nst):
            G = lines[q, n, :, 3]
            y_flame = -1.0
            for j in range(ny - 1):
                G1, G2 = G[j], G[j + 1]
                if (G1 - 0.5) * (G2 - 0.5) <= 0.0:
                    y1, y2 = j * dy, (j + 1) * dy
                    y_flame = y1 if abs(G2 - G1) < 1e-9 else y1 + (0.5 - G1) / (G2 - G1) * (y2 - y1)
                    break
            if not y_flame > 0.0:
                continue
            yp = np.arange(ny) * dy
            yr = yp - y_flame
            keep = np.abs(yr) <= 1.0
            k = int(keep.sum())
            cols["timestep"].append(np.full(k, float(t0 + q)))
            cols["x_location"].append(np.full(k, x_locations[n]))
            cols["y_flame"].append(np.full(k, y_flame))
            cols["y_physical"].append(yp[keep])
            cols["y_relative"].append(yr[keep])
            for c, idx in (("u", 0), ("v", 1), ("w", 2), ("G", 3), ("nu_t", 4), ("S_mag", 5)):
                cols[c].append(lines[q, n, keep, idx])
    return {c: (np.concatenate(v) if v else np.zeros(0)) for c, v in cols.items()}


def read_moments_file(path: str):
    """profile_stats.bin (les_solver_pstat_write): the edges and the moment sums."""
    with open(path, "rb") as f:
        raw = f.read()
    hdr = np.frombuffer(raw[:20], dtype=np.int32)
    if int(hdr[0]) != 0x53505350:
        raise ValueError(f"{path}: not a profile_stats file")
    ny, nrc, nho, npdf = (int(x) for x in hdr[1:])
    vals = np.frombuffer(raw[20:], dtype=np.float64)
    edges, o = {}, 0
    for k, n in (("y_mm", ny), ("g_rc", nrc), ("g_ho", nho), ("u", npdf), ("v", npdf)):
        edges[k] = vals[o:o + n + 1].copy()
        o += n + 1
    sums = vals[o:].copy()
    if len(sums) != moments_size(edges):
        raise ValueError(f"{path}: truncated")
    return edges, sums
