"""Warm-started solves of one SDOT problem at a time, with reusable handles.

``WarmSolver.solve(problem)`` runs the warm-start pipeline:

1. a start: zero on the coarsest level of the problem's multilevel chain
   (``start="multilevel"``); or the learned network's prediction on the
   level of the chain it was trained for (``start="learned"``), either
   averaged down to the coarsest level as that level's start
   (``learned_at="coarsest"``, every level is still solved) or used on its
   own level, which the chain then begins with (``learned_at="level"``);
   or zero on the problem itself (``start="zero"``);
2. every level of the chain from there up, each solved to ``coarse_tol`` by
   this library's damped Newton solve (``cot_solve_newton``) and
   interpolated to the next (``multilevel.prolong``), the finest to ``tol``;
3. the plain L-BFGS (``cot_solve``, COT_SOLVE_WOLFE) from the finest
   level's weights to ``tol``: it evaluates its start and stops at once when
   the tolerance holds, else it finishes the solve, so the plain method
   stays both the fall-back and the judge of the error.

One library handle per level is kept between calls: later problems of the
same sizes reuse their device buffers (``cot_set_problem`` grows them only)
and the trial-loop graph of the L-BFGS.  The reference has no counterpart:
its solver starts from the previous outer iteration's weights or from zero
(main.cu:193-198).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import capi, multilevel
from .problems import SDOTProblem


@dataclass
class WarmStats:
    converged: bool
    max_rel_err: float              # the judge's, at exit
    wall_ms: float                  # host wall time of the whole pipeline
    device_ms: float                # summed device time of the solves
    infer_ms: float = 0.0           # the network's inference (learned start)
    levels: list = field(default_factory=list)   # (n, NewtonStats) per level, coarsest first
    judge: object = None            # the plain L-BFGS's SolveStats
    level_wall_ms: list = field(default_factory=list)   # host wall time per level (prolongation, upload, solve)
    chain_ms: float = 0.0           # host time building the chain (coarsening)


class WarmSolver:
    def __init__(self, start: str = "multilevel", net=None, net_level_sites: int = 0, min_sites: int = 1024,
                 tol: float = 1e-4, coarse_tol: float = 1e-3, history: int = 10, device: int = 0,
                 learned_at: str = "coarsest", shrink_steps: int = 0):
        if start not in ("multilevel", "learned", "zero"):
            raise ValueError(f"unknown start {start!r}")
        if start == "learned" and net is None:
            raise ValueError("a learned start needs the network")
        if learned_at not in ("coarsest", "level"):
            raise ValueError(f"unknown learned_at {learned_at!r}")
        self.learned_at = learned_at
        self.shrink_steps = shrink_steps
        self.start = start
        self.net = net
        self.net_level_sites = net_level_sites
        self.min_sites = min_sites
        self.tol = tol
        self.coarse_tol = coarse_tol
        self.history = history
        self.device = device
        self._handles = {}

    def close(self):
        for s in self._handles.values():
            s.close()
        self._handles = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _handle(self, k: int) -> capi.Solver:
        if k not in self._handles:
            self._handles[k] = capi.Solver(device=self.device)
        return self._handles[k]

    def chain(self, p: SDOTProblem) -> list:
        """The levels this pipeline solves, finest first."""
        if self.start == "zero":
            return [p]
        ch = multilevel.chain(p, self.min_sites)
        if self.start == "learned" and self.learned_at == "level":
            keep = [q for q in ch if q.n >= self.net_level_sites]
            ch = keep if keep else ch[:1]
        return ch

    def _net_level(self, ch) -> int:
        """Index in ``ch`` of the level the network predicts on: the one with
        its training size, else the finest one below it, else the coarsest."""
        for k, q in enumerate(ch):
            if q.n <= self.net_level_sites:
                return k
        return len(ch) - 1

    def solve(self, p: SDOTProblem):
        """(weights of ``p`` in its site order, WarmStats)."""
        t0 = time.perf_counter()
        ch = self.chain(p)
        chain_ms = 1e3 * (time.perf_counter() - t0)
        infer_ms = 0.0
        if self.start == "learned":
            from . import warmstart

            ti = time.perf_counter()
            k = self._net_level(ch)
            w = warmstart.predict(self.net, [ch[k]])[0]
            if k != len(ch) - 1:
                w = multilevel.restrict(w, ch[k], ch[-1])
            infer_ms = 1e3 * (time.perf_counter() - ti)
        else:
            w = np.zeros(ch[-1].n)
        levels = []
        lwall = []
        dev_ms = 0.0
        for k in range(len(ch) - 1, -1, -1):
            tl = time.perf_counter()
            q = ch[k]
            if k < len(ch) - 1:
                w = multilevel.prolong(w, ch[k + 1], q)
            s = self._handle(k)
            s.set_problem(q.xy, q.nu, q.picture, q.size, q.proj_domain)
            w, st = s.solve_newton(w, tol=self.tol if k == 0 else self.coarse_tol, history=self.history,
                                   shrink_steps=self.shrink_steps)
            levels.append((q.n, st))
            lwall.append(1e3 * (time.perf_counter() - tl))
            dev_ms += st.ms
        # the judge: the plain L-BFGS on the finest level's handle
        w, js = self._handle(0).solve(w, mode=capi.SOLVE_WOLFE, tol=self.tol, history=self.history,
                                      max_iter=100000)
        dev_ms += js.ms
        wall = 1e3 * (time.perf_counter() - t0)
        return w, WarmStats(bool(js.converged), js.max_rel_err, wall, dev_ms, infer_ms, levels, js, lwall, chain_ms)
