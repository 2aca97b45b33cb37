"""Multilevel warm start for the SDOT solve.

The dual weights are a smooth function of the site position (w(s) =
|s|^2 - 2 phi(s) for the transport's convex potential phi), so a coarse
problem carries most of their large-scale shape.  ``solve`` builds a chain
of problems, each with 2 x 2 sites merged into one (mean position, summed
mass) and, where the image is fine enough, 2 x 2 pixels merged too.  It
solves the coarsest from w = 0, then each finer one from the weights of
the level below, interpolated bilinearly at its sites, and the finest to
the requested tolerance.  Every level is a plain solve of this library
(cot_solve / cot_solve_batch), so the plain method alone decides when the
error is small enough.  The reference has no counterpart: its solver starts
from the previous weights or zero (main.cu:193-198).

Sites must form a jittered G_x x G_y lattice (``SDOTProblem.grid``), indexed
i = a + G_x b, as the benchmark problems are.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from .problems import SDOTProblem


def _sum2x2(a: np.ndarray) -> np.ndarray:
    """Sums of the 2 x 2 blocks of the first two axes, (a00 + a01) + (a10 +
    a11), by strided adds (several times faster than a reshaped axis sum)."""
    r = a[:, 0::2] + a[:, 1::2]
    return r[0::2] + r[1::2]


def coarsen(p: SDOTProblem, min_pixels_per_site: int = 8) -> SDOTProblem:
    """The problem with each 2 x 2 block of sites merged (mean position,
    summed mass).  The image is merged 2 x 2 as well (pixel masses summed)
    when the unmerged image has at least ``min_pixels_per_site`` pixels
    across a coarse site's pitch (so the merged image keeps at least half
    that many), which makes a coarse evaluation cheaper."""
    gx, gy = p.grid
    if gx % 2 or gy % 2:
        raise ValueError(f"coarsen: site lattice {gx}x{gy} is not even")
    xy = 0.25 * _sum2x2(np.asarray(p.xy, np.float64).reshape(gy, gx, 2)).reshape(-1, 2)
    nu = _sum2x2(np.asarray(p.nu, np.float64).reshape(gy, gx)).ravel()
    W, H = p.size
    pic, size = p.picture, p.size
    if W % 2 == 0 and H % 2 == 0 and W // (gx // 2) >= min_pixels_per_site and H // (gy // 2) >= min_pixels_per_site:
        pic = _sum2x2(np.asarray(p.picture, np.float64).reshape(H, W)).ravel()
        size = (W // 2, H // 2)
    return SDOTProblem(p.name + "/coarse", xy, nu, pic, size, np.array(p.proj_domain, np.float64), (gx // 2, gy // 2))


def prolong(wc: np.ndarray, coarse: SDOTProblem, fine: SDOTProblem) -> np.ndarray:
    """Weights of ``coarse`` interpolated bilinearly at the sites of
    ``fine`` (coarse site (a, b) taken at its lattice point ((a + 0.5) / G_x,
    (b + 0.5) / G_y) of the domain; held constant beyond the outer sites),
    with their mean removed."""
    gxc, gyc = coarse.grid
    Wc = np.asarray(wc, np.float64).ravel()
    d = np.asarray(fine.proj_domain, np.float64)
    x = (fine.xy[:, 0] - d[0]) * (gxc / (d[1] - d[0])) - 0.5
    y = (fine.xy[:, 1] - d[2]) * (gyc / (d[3] - d[2])) - 0.5
    np.clip(x, 0.0, gxc - 1.0, out=x)
    np.clip(y, 0.0, gyc - 1.0, out=y)
    x0 = np.minimum(x.astype(np.int64), max(gxc - 2, 0))   # x >= 0: truncation is the floor
    y0 = np.minimum(y.astype(np.int64), max(gyc - 2, 0))
    fx = x - x0
    fy = y - y0
    i00 = x0 + y0 * gxc
    dx = 1 if gxc > 1 else 0
    dy = gxc if gyc > 1 else 0
    w00, w01, w10, w11 = Wc[i00], Wc[i00 + dx], Wc[i00 + dy], Wc[i00 + dx + dy]
    a = w00 + fx * (w01 - w00)
    b = w10 + fx * (w11 - w10)
    w = a + fy * (b - a)
    return w - w.mean()


def restrict(wf: np.ndarray, fine: SDOTProblem, coarse: SDOTProblem) -> np.ndarray:
    """Weights of ``fine`` averaged over the blocks of sites that make up
    each site of ``coarse`` (a lattice coarser by a power of two per side,
    as ``chain`` builds it), with their mean removed.  A coarse site is the
    mean of its block, and w is smooth in the site position, so the block
    mean is the weight at the coarse site up to the lattice's curvature."""
    gxf, gyf = fine.grid
    gxc, gyc = coarse.grid
    if gxf % gxc or gyf % gyc:
        raise ValueError("restrict: the coarse lattice does not divide the fine one")
    fx, fy = gxf // gxc, gyf // gyc
    w = np.asarray(wf, np.float64).reshape(gyc, fy, gxc, fx).mean(axis=(1, 3)).ravel()
    return w - w.mean()


def chain(p: SDOTProblem, min_sites: int = 1024, max_levels: int = 8) -> list:
    """[p, coarser, ...]: halve the lattice while both sides stay even and
    the next level keeps at least ``min_sites`` sites."""
    out = [p]
    while len(out) <= max_levels:
        gx, gy = out[-1].grid
        if gx % 2 or gy % 2 or (gx // 2) * (gy // 2) < min_sites:
            break
        out.append(coarsen(out[-1]))
    return out


@dataclass
class LevelStats:
    n: int                  # sites of the level
    image: tuple            # its image size
    tol: float              # the max-rel error it was solved to
    stats: list = field(default_factory=list)   # SolveStats (NewtonStats) of each instance
    ms: float = 0.0         # device time of the level's (batched) solve
    judge: list = field(default_factory=list)   # finest level: the plain L-BFGS's SolveStats per instance


def _library_level(level, starts, tol, history, max_iter, batched):
    """One level with this library's solver: (weights, SolveStats list,
    device ms)."""
    from . import capi

    sols = []
    try:
        for q in level:
            sols.append(capi.Solver())
            sols[-1].set_problem(q.xy, q.nu, q.picture, q.size, q.proj_domain)
        if batched:
            ws, st = capi.solve_batch(sols, starts, tol=tol, history=history, max_iter=max_iter)
            return ws, st, st[0].ms
        res = [s.solve(w, mode=capi.SOLVE_WOLFE, tol=tol, history=history, max_iter=max_iter)
               for s, w in zip(sols, starts)]
        st = [r[1] for r in res]
        return [r[0] for r in res], st, float(sum(x.ms for x in st))
    finally:
        for s in sols:
            s.close()


def _newton_level(level, starts, tol, history, max_iter):
    """One level with this library's damped Newton solve (cot_solve_newton),
    instance by instance: (weights, NewtonStats list, device ms)."""
    from . import capi

    ws, sts = [], []
    for q, w in zip(level, starts):
        with capi.Solver() as s:
            s.set_problem(q.xy, q.nu, q.picture, q.size, q.proj_domain)
            wq, st = s.solve_newton(w, tol=tol, history=history)
        ws.append(wq)
        sts.append(st)
    return ws, sts, float(sum(x.ms for x in sts))


def _judge(probs, ws, tol, history):
    """The plain L-BFGS (COT_SOLVE_WOLFE) from each result to ``tol``: it
    evaluates the start and stops at once when the tolerance already holds,
    else it finishes the solve.  Returns (weights, SolveStats list)."""
    from . import capi

    out, sts = [], []
    for q, w in zip(probs, ws):
        with capi.Solver() as s:
            s.set_problem(q.xy, q.nu, q.picture, q.size, q.proj_domain)
            wq, st = s.solve(w, mode=capi.SOLVE_WOLFE, tol=tol, history=history, max_iter=100000)
        out.append(wq)
        sts.append(st)
    return out, sts


def solve(probs: Sequence[SDOTProblem], *, tol: float = 1e-4, coarse_tol: float = 1e-3, min_sites: int = 1024,
          history: int = 10, max_iter: int = 100000, w0: Sequence[np.ndarray] = None, batched: bool = True,
          level_solver=None, method: str = "lbfgs", judge: bool = False):
    """Solve every problem to max-rel error ``tol`` through its multilevel
    chain: the coarsest level from zero (or from ``w0``, one start vector
    per problem of the coarsest level's size), every other level from the
    level below, the coarse levels to ``coarse_tol``.  The problems' chains
    are cut to the shortest one.  With ``method="lbfgs"`` each level runs as
    one batched solve (cot_solve_batch) when ``batched``, else one solve per
    problem; with ``method="newton"`` each level is a damped Newton solve
    (cot_solve_newton) per problem.  ``judge``: the plain L-BFGS then runs
    from the finest level's weights to ``tol`` (it stops at its first
    evaluation when the tolerance holds), so that the plain method decides
    the error; its stats are the last level's ``judge``.
    Returns (weights of the finest level per problem, [LevelStats] from the
    coarsest level up); a level's ``ms`` is its device time (the judge's
    included).

    ``level_solver(problems, starts, tol)``, when given, solves a level in
    place of this library's solver and returns (weights, stats with
    ``iterations`` and ``max_rel_err``, ms)."""
    if method not in ("lbfgs", "newton"):
        raise ValueError(f"unknown method {method!r}")
    chains = [chain(p, min_sites) for p in probs]
    depth = min(len(c) for c in chains)
    chains = [c[:depth] for c in chains]
    ws = list(w0) if w0 is not None else [np.zeros(c[-1].n) for c in chains]
    levels = []
    for k in range(depth - 1, -1, -1):
        level = [c[k] for c in chains]
        if k < depth - 1:
            ws = [prolong(w, c[k + 1], c[k]) for w, c in zip(ws, chains)]
        lt = tol if k == 0 else coarse_tol
        if level_solver is not None:
            ws, st, ms = level_solver(level, ws, lt)
        elif method == "newton":
            ws, st, ms = _newton_level(level, ws, lt, history, max_iter)
        else:
            ws, st, ms = _library_level(level, ws, lt, history, max_iter, batched)
        levels.append(LevelStats(level[0].n, tuple(level[0].size), lt, list(st), ms))
    if judge and level_solver is None:
        ws, jst = _judge([c[0] for c in chains], ws, tol, history)
        levels[-1].judge = jst
        levels[-1].ms += float(sum(x.ms for x in jst))
    return ws, levels
