"""Batches of independent solves on one GPU (the batched configuration of the
solver: 64 instances of uneven N, each with its own target image).

``solve`` puts every instance on its own handle and solves them all in one
CUDA graph launch (``capi.solve_batch``): each instance is a branch of the
graph with its own device-driven trial loop, so small instances run side by
side instead of one after another.  ``autotune`` picks the cell kernel's
shape for a batch -- cells per warp and sites per neighbour bucket -- by
timing short batched runs of a sample of the instances.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import capi, problems

CELLS_PER_WARP = (1, 2, 4)
BUCKET_SIZES = (4, 8, 16)


@dataclass
class TuneResult:
    cells_per_warp: int
    bucket_size: int
    table: List[Tuple[int, int, float]]   # (cells per warp, bucket size, cell-evals/s) per candidate


def instances(count: int = 64, config: int = 3, **kw) -> list:
    """The seeded instances of the batched configuration (N log-uniform in
    [1024, 32768], 512^2 Gaussian-mixture targets); kw shrinks them for tests."""
    return [problems.make(config, i, **kw) for i in range(count)]


def _solvers(probs: Sequence, cells_per_warp: int, bucket_size: int, stream=None) -> list:
    out = []
    for p in probs:
        s = capi.Solver(cells_per_warp=cells_per_warp, bucket_size=bucket_size)
        if stream is not None:
            s.set_stream(stream)
        s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        out.append(s)
    return out


def solve(probs: Sequence, *, cells_per_warp: int = 0, bucket_size: int = 0, stream=None, **opts):
    """Solve every problem from w = 0 in one graph launch.  Returns
    (weights, stats, seconds of the batch as the device timed it)."""
    sol = _solvers(probs, cells_per_warp, bucket_size, stream)
    try:
        ws, st = capi.solve_batch(sol, [np.zeros(p.n) for p in probs], **opts)
    finally:
        for s in sol:
            s.close()
    return ws, st, st[0].ms * 1e-3


def solve_sequential(probs: Sequence, *, cells_per_warp: int = 0, bucket_size: int = 0, stream=None, **opts):
    """The same solves one after another on one handle each (the baseline the
    batch is measured against).  Returns (weights, stats, summed seconds)."""
    ws, st = [], []
    for p in probs:
        (s,) = _solvers([p], cells_per_warp, bucket_size, stream)
        try:
            w, x = s.solve(np.zeros(p.n), **opts)
        finally:
            s.close()
        ws.append(w)
        st.append(x)
    return ws, st, sum(x.ms for x in st) * 1e-3


def autotune(probs: Sequence, *, sample: int = 8, max_iter: int = 60, stream=None,
             cells_per_warp=CELLS_PER_WARP, bucket_sizes=BUCKET_SIZES, **opts) -> TuneResult:
    """Time a short batched run (max_iter iterations) of an evenly spread
    sample of the instances under every candidate shape and keep the one with
    the highest cell-evaluation rate."""
    order = np.argsort([p.n for p in probs])
    pick = [probs[int(order[k])] for k in np.linspace(0, len(probs) - 1, min(sample, len(probs))).astype(int)]
    table = []
    for cpw, bs in itertools.product(cells_per_warp, bucket_sizes):
        # once to settle allocations, once timed
        solve(pick, cells_per_warp=cpw, bucket_size=bs, stream=stream, max_iter=max_iter, **opts)
        _, st, sec = solve(pick, cells_per_warp=cpw, bucket_size=bs, stream=stream, max_iter=max_iter, **opts)
        rate = sum(p.n * x.evaluations for p, x in zip(pick, st)) / max(sec, 1e-9)
        table.append((cpw, bs, rate))
    best = max(table, key=lambda r: r[2])
    return TuneResult(best[0], best[1], table)
