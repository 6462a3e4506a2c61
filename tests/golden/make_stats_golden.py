#!/usr/bin/env python3
"""Generate the golden profile statistics from the reference's own post-processing code.

Writes a seeded synthetic probe file in the solver's CSV layout, then runs on it
  * bayesian_optimizer.load_and_compute_reynolds_stress (returns the G-binned <u'v'>),
  * analysis.task_1_3_flame_profile and analysis.task_1_6_reynolds_stress_vs_g_binned,
    whose profiles are the arguments they hand to the plotting calls;
and, for the optimiser, bayesian_optimizer's experimental_reynolds_stress, smooth_profile,
compute_score (on seeded profiles) and BayesianOptimizer._acquisition / suggest_next (on a
seeded history, with numpy's global generator seeded before each call);
with stand-in matplotlib / seaborn modules that record those plotting calls (neither
library is installed here).  The reference modules are imported from their source tree,
unmodified.  Output: ``tests/golden/stats_ref.npz`` holding the probe file's text
(``csv_text``, uint8) and the reference's profiles.

Usage: python tests/golden/make_stats_golden.py [reference_dir]
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
import build_ref  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else build_ref.default_ref()


class Recorder:
    """Stands in for figures, axes and pyplot; records every .plot(x, y, ...) call."""

    calls = []

    def __init__(self, tag="obj"):
        self.tag = tag

    def plot(self, *a, **k):
        Recorder.calls.append((self.tag, [np.asarray(x, dtype=np.float64) for x in a[:2]], k.get("label")))
        return [Recorder()]

    def __getattr__(self, name):
        return lambda *a, **k: Recorder(name)

    def __getitem__(self, i):
        return Recorder(f"{self.tag}[{i}]")


def _subplots(nrows=1, ncols=1, **k):
    n = nrows * ncols
    axes = np.empty(n, dtype=object)
    for q in range(n):
        axes[q] = Recorder(f"ax{q}")
    return Recorder("fig"), (axes if n > 1 else axes[0])


def install_stubs():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    plt.rcParams = {}
    plt.subplots = _subplots
    for name in ("switch_backend", "tight_layout", "savefig", "close", "figure", "hist", "title", "xlabel", "ylabel",
                 "grid", "legend", "scatter", "colorbar", "axhline", "axvline", "yscale", "xlim", "ylim", "text",
                 "plot", "subplot", "suptitle"):
        setattr(plt, name, lambda *a, **k: Recorder())
    mpl.pyplot = plt
    cm = types.ModuleType("matplotlib.cm")
    colors = types.ModuleType("matplotlib.colors")
    colors.LogNorm = lambda *a, **k: None
    colors.Normalize = lambda *a, **k: None
    mpl.cm, mpl.colors = cm, colors
    sns = types.ModuleType("seaborn")
    sns.kdeplot = lambda *a, **k: Recorder()
    sns.histplot = lambda *a, **k: Recorder()
    sys.modules.update({"matplotlib": mpl, "matplotlib.pyplot": plt, "matplotlib.cm": cm,
                        "matplotlib.colors": colors, "seaborn": sns})


def synthetic_probe_rows(seed=7, steps=300, ny=48, dy=0.064 / 48):
    """Rows shaped like the solver's: a wrinkled flame front at y_flame(t), G rising across it
    from 0 to 1 (clipped, with exact 0s and 1s), velocities correlated with G and noise."""
    rng = np.random.default_rng(seed)
    rows = []
    for t in range(steps):
        y_flame = 0.02 + 0.004 * np.sin(0.05 * t) + 0.001 * rng.standard_normal()
        for j in range(ny):
            yp = j * dy
            yr = yp - y_flame
            G = float(np.clip(0.5 + yr / 0.006 + 0.05 * rng.standard_normal(), 0.0, 1.0))
            u = 5.0 + 6.0 * G + 0.6 * rng.standard_normal()
            v = 0.3 * (G - 0.5) + 0.4 * rng.standard_normal() + 0.2 * (u - 5.0 - 6.0 * G)
            w = 0.35 * rng.standard_normal()
            rows.append((t, 0.035, y_flame, yp, yr, u, v, w, G, 1e-5 * (1 + G), 100.0 * (1 + rng.random())))
    return rows


def write_csv(path, rows):
    with open(path, "w") as fp:
        fp.write("timestep,x_location,y_flame,y_physical,y_relative,u,v,w,G,nu_t,S_mag\n")
        for r in rows:
            fp.write("%d,%.3f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6f,%.6e,%.6e\n" % r)


def main():
    install_stubs()
    sys.path.insert(0, REF)
    bo = importlib.import_module("bayesian_optimizer")
    an = importlib.import_module("analysis")
    import pandas as pd

    out = {}
    with tempfile.TemporaryDirectory() as d:
        csv_path = os.path.join(d, "probe_data_flame_region_loc0.csv")
        write_csv(csv_path, synthetic_probe_rows())
        out["csv_text"] = np.frombuffer(open(csv_path, "rb").read(), dtype=np.uint8)
        df = pd.read_csv(csv_path)
        g, s = bo.load_and_compute_reynolds_stress(d, loc_index=0, num_bins=20)
        out["uv_G_centers"], out["uv_stress"] = np.asarray(g), np.asarray(s)
        g, s = bo.load_and_compute_reynolds_stress(d, loc_index=0, num_bins=37)
        out["uv37_G_centers"], out["uv37_stress"] = np.asarray(g), np.asarray(s)
    Recorder.calls = []
    an.task_1_3_flame_profile(df, "/nonexistent")
    for tag, (x, y), label in Recorder.calls:
        out[f"flame_profile.{label}.x"], out[f"flame_profile.{label}.y"] = x, y
    Recorder.calls = []
    an.task_1_6_reynolds_stress_vs_g_binned(df, "/nonexistent")
    names = ["uu_cond", "vv_cond", "uv_cond"]
    for q, (tag, (x, y), label) in enumerate(Recorder.calls):
        out[f"stress_vs_G.{names[q]}.x"], out[f"stress_vs_G.{names[q]}.y"] = x, y
    # ---- optimiser pieces
    rng = np.random.default_rng(11)
    g = np.linspace(0.0, 1.0, 41)
    out["exp_G"], out["exp_val"] = g, bo.experimental_reynolds_stress(g)
    profiles = []
    for q in range(6):
        centers = 0.5 * (np.linspace(0, 1, 21)[:-1] + np.linspace(0, 1, 21)[1:])
        val = 0.02 * np.exp(-(3 + 5 * q) * centers) + 0.002 * rng.standard_normal(20)
        val[rng.random(20) < 0.15 * q] = np.nan
        profiles.append(val)
    out["prof_G"] = centers
    out["prof_val"] = np.array(profiles)
    out["prof_score"] = np.array([bo.compute_score(centers, p) for p in profiles])
    sm = [bo.smooth_profile(centers[~np.isnan(p)], p[~np.isnan(p)]) for p in profiles[:3]]
    out["smooth_G"] = np.array([a for a, b in sm])
    out["smooth_val"] = np.array([b for a, b in sm])
    out["uv_score"] = np.array([bo.compute_score(out["uv_G_centers"], out["uv_stress"])])
    with tempfile.TemporaryDirectory() as d:
        opt = bo.BayesianOptimizer(history_file=os.path.join(d, "h.json"))
        lo, hi = opt.bounds[:, 0], opt.bounds[:, 1]
        X = rng.uniform(lo, hi, size=(12, 6))
        y = np.array([float(np.sum(((x - lo) / (hi - lo) - 0.4) ** 2)) for x in X])
        opt.X_obs, opt.y_obs = [list(map(float, x)) for x in X], list(map(float, y))
        np.random.seed(5)
        Xc = np.random.uniform(lo, hi, size=(300, 6))
        np.random.seed(6)
        out["ei"] = opt._acquisition(Xc)
        out["ei_X"], out["ei_y"], out["ei_cand"] = X, y, Xc
        np.random.seed(9)
        nxt = opt.suggest_next(n_candidates=500)
        out["next"] = np.array([nxt[k] for k in opt.param_names])
    np.savez_compressed(os.path.join(HERE, "stats_ref.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
