"""Comparison helpers for the tests that run the reference solver beside the GPU solver:
probe files (les_combustion_solver.c:3403-3471, rows printed with %.6f and %.6e) and the
monitor file (:3874-3918, %.6e / %.2f / %.4f / %.2e).  Printed values can differ by at most
one unit of their last digit when the underlying doubles agree to rounding level."""
import os

import numpy as np


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def parse_probe(text):
    rows = [ln.split(",") for ln in text.splitlines()[1:] if ln.strip()]
    return np.array([[float(x) for x in r] for r in rows]).reshape(-1, 11)


def compare_probes(gpu_texts, ref_texts):
    """Both dicts map station -> file text (or None).  Asserts the same rows, values within
    one unit of the last printed digit; returns the largest fixed-point difference."""
    worst = 0.0
    for n in range(7):
        a_txt, b_txt = gpu_texts.get(n), ref_texts.get(n)
        if b_txt is None:
            assert a_txt is None, f"station {n}: GPU wrote rows the reference did not"
            continue
        assert a_txt is not None, f"station {n}: no GPU rows"
        a, b = parse_probe(a_txt), parse_probe(b_txt)
        assert a.shape == b.shape, f"station {n}: {a.shape[0]} rows against the reference's {b.shape[0]}"
        d_fixed = np.abs(a[:, :9] - b[:, :9]).max(initial=0.0)
        assert d_fixed <= 1.01e-6, f"station {n}: fixed-point columns differ by {d_fixed:.3e}"
        scale = np.maximum(np.abs(b[:, 9:]), 1e-300)
        d_exp = (np.abs(a[:, 9:] - b[:, 9:]) / scale).max(initial=0.0)
        assert d_exp <= 1.01e-6, f"station {n}: nu_t/S_mag differ by {d_exp:.3e} relative"
        worst = max(worst, d_fixed)
    return worst


def read_probe_texts(directory):
    out = {}
    for n in range(7):
        p = os.path.join(directory, f"probe_data_flame_region_loc{n}.csv")
        if os.path.exists(p):
            with open(p) as f:
                out[n] = f.read()
    return out


def compare_monitor(a_txt, b_txt):
    """step,dt,total_mass,min_T,max_T,min_G,max_G,min_Y_C3H8 rows: the same steps, each value
    within one unit of its printed last digit (relative 1e-6 for the %e columns, 0.01 for T
    at %.2f, 1e-4 for G at %.4f, relative 1e-2 for %.2e)."""
    a = [ln.split(",") for ln in a_txt.splitlines()[1:] if ln.strip()]
    b = [ln.split(",") for ln in b_txt.splitlines()[1:] if ln.strip()]
    assert len(a) == len(b) > 0, (len(a), len(b))
    A = np.array([[float(x) for x in r] for r in a])
    B = np.array([[float(x) for x in r] for r in b])
    assert (A[:, 0] == B[:, 0]).all()
    for c, kind, tol in ((1, "rel", 1.01e-6), (2, "rel", 1.01e-6), (3, "abs", 0.0101), (4, "abs", 0.0101),
                         (5, "abs", 1.01e-4), (6, "abs", 1.01e-4), (7, "rel", 1.01e-2)):
        d = np.abs(A[:, c] - B[:, c])
        if kind == "rel":
            d = d / np.maximum(np.abs(B[:, c]), 1e-300)
        assert d.max() <= tol, f"monitor column {c}: {d.max():.3e}"
