#!/usr/bin/env python3
"""Generate the golden fixtures from the reference solver itself.

Runs the compiled reference (``oracle/_ref/<config>/les_ref``, built by
``oracle/build_ref.py`` from the reference source) with OMP_NUM_THREADS=1 and stores, for
each case, the state after every dumped step, the dt sequence, the probe CSV texts and the
monitor CSV text in ``tests/golden/<case>.npz``.  The fixtures pin the oracle and the GPU
solver on machines where the reference source is not available.

Cases (seed 1234 unless noted):
  tiny_s10     24x12x16 grid, 10 steps from t_loop = 0 (states after steps 1 and 10)
  tiny_w495    24x12x16 grid, 10 steps from t_loop = 495 (crosses the WENO-gradient switch;
               state after step 10)
  small_s12    40x16x24 grid, 12 steps, state after step 12, seed 77
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_ref  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "tiny_s10": dict(config="tiny", steps=10, start=0, seed=1234, keep=[1, 10]),
    "tiny_w495": dict(config="tiny", steps=10, start=495, seed=1234, keep=[10]),
    "small_s12": dict(config="small", steps=12, start=0, seed=77, keep=[12]),
}
FIELDS = build_ref.STATE_FIELDS


def make(name: str, spec: dict) -> str:
    if not oracle.ref_available(spec["config"]):
        build_ref.build(build_ref.default_ref(), [spec["config"]])
    dumps, meta = oracle.run_reference(spec["config"], spec["steps"], seed=spec["seed"], start=spec["start"],
                                       dump_every=1)
    out = {"steps": np.array(spec["keep"]), "dt": np.array([dumps[n]["dt"] for n in range(1, spec["steps"] + 1)]),
           "seed": np.array(spec["seed"]), "start": np.array(spec["start"])}
    for n in spec["keep"]:
        for f in FIELDS:
            out[f"s{n}_{f}"] = dumps[n][f]
    for k, txt in meta["probes"].items():
        out[f"probe{k}"] = np.frombuffer(txt.encode(), dtype=np.uint8)
    out["monitor"] = np.frombuffer(meta["monitor"].encode(), dtype=np.uint8)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, config=np.array(spec["config"]), **out)
    return path


def main() -> int:
    for name, spec in CASES.items():
        p = make(name, spec)
        print(p, os.path.getsize(p))
    return 0


if __name__ == "__main__":
    sys.exit(main())
