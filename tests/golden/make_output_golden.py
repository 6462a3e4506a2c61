#!/usr/bin/env python3
"""Golden output files from the reference solver itself (``oracle/_ref``, built from its
source by ``oracle/build_ref.py``): the VTK file of the last step and the point time series.

  tiny  (24x12x16), seed 1234, 10 steps: Premixed_C3H8_Air_0010.vtk (output_vtk at the end
        of the run, :4611)
  small (40x16x24), seed 77, 60 steps: LES_point_data_phi*_i*_j*_k*.csv (flushed at step 50
        and at the end of the run, :4587, :4621)

Stored as the files' bytes in ``tests/golden/outputs_ref.npz``.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402


def main():
    out = {}
    with tempfile.TemporaryDirectory() as d:
        w = os.path.join(d, "tiny")
        oracle.run_reference("tiny", 10, seed=1234, dump_every=0, keep_dir=w, novtk=False)
        vtk = os.path.join(w, "Premixed_C3H8_Air_0010.vtk")
        out["vtk_tiny_s10"] = np.frombuffer(open(vtk, "rb").read(), dtype=np.uint8)
        w = os.path.join(d, "small")
        oracle.run_reference("small", 60, seed=77, dump_every=0, keep_dir=w, novtk=True)
        names = sorted(f for f in os.listdir(w) if f.startswith("LES_point_data"))
        out["point_names"] = np.array(names)
        for q, f in enumerate(names):
            out[f"point_{q}"] = np.frombuffer(open(os.path.join(w, f), "rb").read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "outputs_ref.npz"), **out)
    print(sorted(out), [len(out[k]) for k in out if k.startswith("point_") or k.startswith("vtk")])


if __name__ == "__main__":
    main()
