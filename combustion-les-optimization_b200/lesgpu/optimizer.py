"""Bayesian optimisation of the model constants, closed over the batched ensemble.

The reference scores one LES at a time against an experimental Reynolds-stress fit and asks
a Gaussian-process model for the next set of six constants, which the user pastes into the C
source as #defines and recompiles (bayesian_optimizer.py:40-64, :421-561, :568-716).  Here
the constants are runtime fields of the solver config, so a round proposes a *batch* of sets
(expected improvement with the kriging-believer heuristic: each proposal's predicted mean is
added as a pseudo-observation before the next), runs them together as one ensemble on the
GPU, scores each member's probe file and updates the model.

Restated from the reference (same formulas, same parameter bounds, same GP model):
  experimental_reynolds_stress  bayesian_optimizer.py:40-64
  smooth_profile                :421-470
  compute_score                 :473-561
  BayesianOptimizer             :568-700 (EI acquisition, random-candidate search)
The GP regression itself is scikit-learn's GaussianProcessRegressor, as in the reference.
"""
from __future__ import annotations

import json
import os
import tempfile
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import stats

PARAM_BOUNDS = {
    "FLAME_ACCEL_STRENGTH": (0.1, 5.0),
    "FLAME_ACCEL_WIDTH": (0.05, 0.30),
    "FLAME_ACCEL_CENTER": (0.40, 0.80),
    "CS_UNBURNED": (0.08, 0.20),
    "CS_BURNT": (0.30, 0.70),
    "CS_FLAME_BOOST": (0.10, 0.40),
}
# the SolverConfig field each optimised constant sets
CONFIG_FIELD = {
    "FLAME_ACCEL_STRENGTH": "accel_strength",
    "FLAME_ACCEL_WIDTH": "accel_width",
    "FLAME_ACCEL_CENTER": "accel_center",
    "CS_UNBURNED": "cs_unburned",
    "CS_BURNT": "cs_burnt",
    "CS_FLAME_BOOST": "cs_flame_boost",
}


def experimental_reynolds_stress(G):
    """The experimental <u'v'>(G) fit: 0.020 exp(-15 G) + 0.005 exp(-1.5 G)."""
    G = np.atleast_1d(np.array(G, dtype=float))
    return 0.020 * np.exp(-15.0 * G) + 0.005 * np.exp(-1.5 * G)


def smooth_profile(G_v, sim_v, n_points: int = 50, smooth_window: int = 5):
    """Average duplicate G values, interpolate with a cubic interpolating spline (linear if
    that fails) onto n_points uniform points, then a moving average of smooth_window points
    with edge padding."""
    from scipy.interpolate import UnivariateSpline
    G_v = np.asarray(G_v, dtype=float)
    sim_v = np.asarray(sim_v, dtype=float)
    uniq, inv = np.unique(G_v, return_inverse=True)
    s_sorted = np.bincount(inv, weights=sim_v) / np.bincount(inv)
    G_sorted = uniq
    if len(G_sorted) < 4:
        return G_sorted, s_sorted
    try:
        spl = UnivariateSpline(G_sorted, s_sorted, k=3, s=0, ext=3)
    except Exception:
        spl = UnivariateSpline(G_sorted, s_sorted, k=1, s=0, ext=3)
    G_uniform = np.linspace(G_sorted[0], G_sorted[-1], n_points)
    sim_interp = spl(G_uniform)
    w = smooth_window
    kernel = np.ones(w) / w
    sim_padded = np.pad(sim_interp, w // 2, mode="edge")
    return G_uniform, np.convolve(sim_padded, kernel, mode="valid")


def compute_score(G_centers, stress_sim, smooth_window: int = 5) -> float:
    """Score of a simulated <u'v'>(G) profile (smaller is better): 5 x the summed increases of
    the smoothed curve + 2 x (1 - its correlation with the experimental fit) + the shortfall
    of its range against the fit's; 1e6 with fewer than 5 valid bins."""
    G_centers = np.asarray(G_centers, dtype=float)
    stress_sim = np.asarray(stress_sim, dtype=float)
    valid = ~np.isnan(stress_sim)
    if valid.sum() < 5:
        return 1e6
    G_smooth, sim_smooth = smooth_profile(G_centers[valid], stress_sim[valid], smooth_window=smooth_window)
    exp_smooth = experimental_reynolds_stress(G_smooth)
    increase_penalty = float(np.sum(np.maximum(0.0, np.diff(sim_smooth))))
    sim_std, exp_std = sim_smooth.std(), exp_smooth.std()
    if sim_std < 1e-10 or exp_std < 1e-10:
        shape_score = 1.0
    else:
        corr = float(np.clip(np.corrcoef(sim_smooth, exp_smooth)[0, 1], -1.0, 1.0))
        shape_score = 1.0 - corr
    sim_range = float(sim_smooth.max() - sim_smooth.min())
    exp_range = float(exp_smooth.max() - exp_smooth.min())
    range_score = max(0.0, 1.0 - sim_range / (exp_range + 1e-10))
    return 5.0 * increase_penalty + 2.0 * shape_score + 1.0 * range_score


class BayesianOptimizer:
    """GP (constant x Matern 5/2, alpha 1e-6, normalised targets, 5 optimiser restarts) over
    the six constants normalised to [0, 1]; expected improvement (xi = 0.01) over uniform
    random candidates.  Random draws come from numpy's global generator unless ``rng`` is
    given."""

    def __init__(self, history_file: Optional[str] = None, rng: Optional[np.random.Generator] = None):
        from sklearn.gaussian_process import GaussianProcessRegressor
        from sklearn.gaussian_process.kernels import ConstantKernel, Matern
        self.param_names = list(PARAM_BOUNDS)
        self.bounds = np.array([PARAM_BOUNDS[k] for k in self.param_names])
        self.history_file = history_file
        self.rng = rng
        self.gp = GaussianProcessRegressor(kernel=ConstantKernel(1.0) * Matern(nu=2.5), alpha=1e-6,
                                           normalize_y=True, n_restarts_optimizer=5)
        self.X_obs: List[List[float]] = []
        self.y_obs: List[float] = []
        if history_file and os.path.exists(history_file):
            with open(history_file) as f:
                data = json.load(f)
            self.X_obs, self.y_obs = data.get("X", []), data.get("y", [])

    def _uniform(self, size=None):
        lo, hi = self.bounds[:, 0], self.bounds[:, 1]
        if self.rng is not None:
            return self.rng.uniform(lo, hi, size=size)
        return np.random.uniform(lo, hi, size=size)

    def _normalize(self, x):
        return (np.asarray(x) - self.bounds[:, 0]) / (self.bounds[:, 1] - self.bounds[:, 0])

    def _fit(self, X, y):
        self.gp.fit(np.array([self._normalize(x) for x in X]), y)

    def expected_improvement(self, X_cand, xi: float = 0.01, X=None, y=None):
        """EI of each candidate for minimisation, after fitting the GP to (X, y) (default: the
        observations).  Uniform random values with fewer than two observations."""
        from scipy.stats import norm
        X = self.X_obs if X is None else X
        y = self.y_obs if y is None else y
        if len(y) < 2:
            return np.random.rand(len(X_cand)) if self.rng is None else self.rng.random(len(X_cand))
        self._fit(X, y)
        mu, sigma = self.gp.predict(np.array([self._normalize(x) for x in X_cand]), return_std=True)
        y_best = np.min(y)
        z = (y_best - mu - xi) / (sigma + 1e-9)
        ei = (y_best - mu - xi) * norm.cdf(z) + sigma * norm.pdf(z)
        ei[sigma < 1e-10] = 0.0
        return ei

    def suggest_next(self, n_candidates: int = 10000) -> Dict[str, float]:
        if len(self.y_obs) < 3:
            return dict(zip(self.param_names, self._uniform()))
        X_cand = self._uniform(size=(n_candidates, len(self.param_names)))
        return dict(zip(self.param_names, X_cand[int(np.argmax(self.expected_improvement(X_cand)))]))

    def suggest_batch(self, q: int, n_candidates: int = 10000) -> List[Dict[str, float]]:
        """q proposals for one ensemble round: the first as suggest_next; each further one
        after adding the previous proposal with the GP's predicted mean as an observation
        (kriging believer), so the batch spreads over distinct promising regions."""
        X, y = list(self.X_obs), list(self.y_obs)
        out = []
        for _ in range(q):
            if len(y) < 3:
                x = self._uniform()
            else:
                X_cand = self._uniform(size=(n_candidates, len(self.param_names)))
                x = X_cand[int(np.argmax(self.expected_improvement(X_cand, X=X, y=y)))]
            out.append(dict(zip(self.param_names, x)))
            if len(y) >= 2:
                self._fit(X, y)
                y.append(float(self.gp.predict(self._normalize(x)[None, :])[0]))
            else:
                y.append(float(np.mean(y)) if y else 0.0)
            X.append(list(map(float, x)))
        return out

    def register_result(self, params: Dict[str, float], score: float):
        self.X_obs.append([float(params[k]) for k in self.param_names])
        self.y_obs.append(float(score))
        if self.history_file:
            with open(self.history_file, "w") as f:
                json.dump({"X": self.X_obs, "y": self.y_obs}, f, indent=2)

    def best_result(self):
        if not self.y_obs:
            return None, None
        b = int(np.argmin(self.y_obs))
        return dict(zip(self.param_names, self.X_obs[b])), self.y_obs[b]


def config_for(base, params: Dict[str, float]):
    """The solver config of one proposal: ``base`` with the six constants replaced."""
    return base.replace(**{CONFIG_FIELD[k]: float(v) for k, v in params.items()})


def score_run(directory: str, loc: int = 0, num_bins: int = 20) -> float:
    """compute_score of the <u'v'>(G) profile of one run's probe file at station ``loc``."""
    path = os.path.join(directory, f"probe_data_flame_region_loc{loc}.csv")
    if not os.path.exists(path):
        return 1e6
    G, s = stats.uv_vs_g(stats.read_probe_csv(path), num_bins)
    return compute_score(G, s)


def run_campaign(base, rounds: int, batch: int, steps: int, precision=None, workdir: Optional[str] = None,
                 loc: int = 0, seed: int = 0, chunk: int = 64, log=print) -> BayesianOptimizer:
    """``rounds`` rounds of ``batch`` proposals, each round one GPU ensemble of ``steps`` steps
    from the initial state, scored from the probe files; returns the optimiser."""
    from . import native as N
    from .ensemble import Ensemble
    precision = N.FP32 if precision is None else precision
    workdir = workdir or tempfile.mkdtemp(prefix="lesopt_")
    opt = BayesianOptimizer(os.path.join(workdir, "optimization_history.json"), rng=np.random.default_rng(seed))
    for r in range(rounds):
        props = opt.suggest_batch(batch)
        cfgs = [config_for(base, p) for p in props]
        ens = Ensemble(cfgs, precision=precision, autotune=False)
        dirs = []
        for q, m in enumerate(ens.members):
            d = os.path.join(workdir, f"round{r:03d}_trial{q:03d}")
            os.makedirs(d, exist_ok=True)
            m.set_outputs(d, N.LES_OUT_PROBES)
            dirs.append(d)
        ens.run(steps, chunk=chunk)
        ens.close()
        for p, d in zip(props, dirs):
            opt.register_result(p, score_run(d, loc))
        best, score = opt.best_result()
        log(f"round {r}: best score {score:.6f}")
    return opt


def main(argv=None) -> int:
    import argparse
    import sys
    from .config import preset
    ap = argparse.ArgumentParser(description="Bayesian optimisation of the model constants over GPU ensembles")
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--rounds", type=int, default=4)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    from . import native as N
    opt = run_campaign(preset(a.workload), a.rounds, a.batch, a.steps,
                       N.FP32 if a.precision == "fp32" else N.FP64, a.workdir, seed=a.seed)
    best, score = opt.best_result()
    print(json.dumps({"best": best, "score": score, "trials": len(opt.y_obs)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
