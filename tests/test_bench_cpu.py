"""The bench's figures that come from the committed ncu summary: the issue
roofline and the live DRAM traffic of the cell kernels (no GPU)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_committed_profile_carries_the_bench_figures():
    b = _bench()
    insts = b.committed_figure("warp_instructions_per_launch")
    traffic = b.committed_traffic()
    # warp instructions of the five cell kernels per evaluation, and their
    # DRAM bytes: both per 65,536-cell evaluation, both positive
    assert insts is not None and 1e8 < insts < 1e9
    assert traffic is not None and 1e5 < traffic < 1e8
    assert b.committed_figure("no_such_key") is None
