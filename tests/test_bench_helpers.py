"""bench.py's byte accounting and the DRAM traffic it reads from the committed ncu summaries
(no GPU): the algorithmic bytes per cell of each kernel class, and the measured per-launch
traffic of the stage kernels at 256x128x128 staying at them (within 1 %) stage by stage."""
import importlib.util
import os

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_algorithmic_bytes_per_cell():
    b = _bench()
    assert b.kernel_bytes_per_cell("rhs_scalar", 8) == 504
    assert b.kernel_bytes_per_cell("filter_props", 8) == 240
    assert b.kernel_bytes_per_cell("strain", 8) == 88 and b.kernel_bytes_per_cell("rhs_flow", 8) == 96
    assert b.kernel_bytes_per_cell("rhs_scalar", 4) == 307
    assert b.kernel_bytes_per_cell("filter_props", 4) == 131
    assert b.STEP_BYTES_PER_CELL == 52 * 4 * 8
    # a stage kernel's launch is credited with one stage's share of the whole-step figure
    assert set(b.STAGE_KERNELS) == {"filter_props", "strain", "rhs_flow", "rhs_scalar"}
    assert b.STEP_BYTES_PER_CELL * 8 / 8 / 4 == 416


def test_committed_traffic_covers_the_stage_kernels():
    b = _bench()
    t = b._traffic_table()
    for prec, e in (("fp64", 8), ("fp32", 4)):
        got = [t[(k, "c2", prec)] for k in ("filter_props", "strain", "rhs_flow", "rhs_scalar")]
        alg = [b.kernel_bytes_per_cell(k, e) for k in ("filter_props", "strain", "rhs_flow", "rhs_scalar")]
        assert all(g > 0 for g in got)
        # a stage moves no more DRAM bytes than its passes' own field counts (halos from L1/L2,
        # no re-reads), within 1 % for the write-back of dirty lines across stages
        assert sum(got) <= 1.01 * sum(alg)
