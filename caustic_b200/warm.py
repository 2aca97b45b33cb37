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
and the trial-loop graph of the L-BFGS.  The problem is copied to the GPU
once; the coarser levels are built there (2 x 2 sums of sites, masses and
pixels), the weights are interpolated there, and every level is handed to
the library as device arrays, so that only the final weights come back.  The reference has no counterpart:
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
class Level:
    """Sizes of one level of a chain (its arrays live on the device)."""
    n: int
    grid: tuple
    size: tuple
    proj_domain: np.ndarray


def chain_shapes(p: SDOTProblem, min_sites: int = 1024, max_levels: int = 8, min_pixels_per_site: int = 8) -> list:
    """The levels multilevel.chain would build, sizes only, finest first."""
    gx, gy = p.grid
    W, H = p.size
    out = [Level(p.n, (gx, gy), (W, H), np.asarray(p.proj_domain, np.float64))]
    while len(out) <= max_levels:
        if gx % 2 or gy % 2 or (gx // 2) * (gy // 2) < min_sites:
            break
        if W % 2 == 0 and H % 2 == 0 and W // (gx // 2) >= min_pixels_per_site and H // (gy // 2) >= min_pixels_per_site:
            W, H = W // 2, H // 2
        gx, gy = gx // 2, gy // 2
        out.append(Level(gx * gy, (gx, gy), (W, H), out[0].proj_domain))
    return out


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
                 learned_at: str = "coarsest", shrink_steps: int = 0, shrink_coarsest: int = 0):
        if start not in ("multilevel", "learned", "zero"):
            raise ValueError(f"unknown start {start!r}")
        if start == "learned" and net is None:
            raise ValueError("a learned start needs the network")
        if learned_at not in ("coarsest", "level"):
            raise ValueError(f"unknown learned_at {learned_at!r}")
        self.learned_at = learned_at
        self.shrink_steps = shrink_steps          # scaled-down starts tried on every level
        self.shrink_coarsest = shrink_coarsest    # ... and on the coarsest level only
        self.start = start
        self.net = net
        self.net_level_sites = net_level_sites
        self.min_sites = min_sites
        self.tol = tol
        self.coarse_tol = coarse_tol
        self.history = history
        self.device = device
        self._handles = {}
        self._stream = None

    def close(self):
        for s in self._handles.values():
            s.close()
        self._handles = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _torch_stream(self):
        """One stream for everything a solve does, the library's work and the
        torch operations around it (levels, prolongation, inference), so that
        each reads what the one before wrote."""
        if self._stream is None:
            import torch

            self._stream = torch.cuda.Stream(device=torch.device("cuda", self.device))
        return self._stream

    def _handle(self, k: int) -> capi.Solver:
        if k not in self._handles:
            s = capi.Solver(device=self.device)
            s.set_stream(self._torch_stream().cuda_stream)
            self._handles[k] = s
        return self._handles[k]

    def chain(self, p: SDOTProblem) -> list:
        """The levels this pipeline solves, finest first."""
        if self.start == "zero":
            return [p]
        ch = chain_shapes(p, self.min_sites)
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

    def _device_chain(self, p: SDOTProblem):
        """The chain's levels as device arrays: (descriptor, xy, nu,
        picture) per level, finest first; the descriptors are SDOTProblems
        without arrays (sizes, grid, domain)."""
        import torch

        dev = torch.device("cuda", self.device)
        gx, gy = p.grid
        W, H = p.size
        xy = torch.from_numpy(np.ascontiguousarray(p.xy, np.float64)).to(dev).view(gy, gx, 2)
        nu = torch.from_numpy(np.ascontiguousarray(p.nu, np.float64)).to(dev).view(gy, gx)
        pic = torch.from_numpy(np.ascontiguousarray(p.picture, np.float64)).to(dev).view(H, W)
        descs = self.chain(p)   # sizes only: the same rules as multilevel.chain
        out = []
        for k, q in enumerate(descs):
            if k > 0:
                # the 2 x 2 sums of multilevel.coarsen, in the same order
                def s2(a):
                    r = a[:, 0::2] + a[:, 1::2]
                    return r[0::2] + r[1::2]

                xy = 0.25 * s2(xy)
                nu = s2(nu)
                if tuple(q.size) != tuple(descs[k - 1].size):
                    pic = s2(pic)
            out.append((q, xy.reshape(-1).contiguous(), nu.reshape(-1).contiguous(), pic.reshape(-1).contiguous()))
        return out

    @staticmethod
    def _prolong(w, coarse, fine_xy, fine):
        """multilevel.prolong on device arrays."""
        import torch

        gxc, gyc = coarse.grid
        d = np.asarray(fine.proj_domain, np.float64)
        xy = fine_xy.view(-1, 2)
        x = ((xy[:, 0] - d[0]) * (gxc / (d[1] - d[0])) - 0.5).clamp_(0.0, gxc - 1.0)
        y = ((xy[:, 1] - d[2]) * (gyc / (d[3] - d[2])) - 0.5).clamp_(0.0, gyc - 1.0)
        x0 = torch.clamp(x.to(torch.int64), max=max(gxc - 2, 0))
        y0 = torch.clamp(y.to(torch.int64), max=max(gyc - 2, 0))
        fx = x - x0
        fy = y - y0
        i00 = x0 + y0 * gxc
        dx = 1 if gxc > 1 else 0
        dy = gxc if gyc > 1 else 0
        w00, w01, w10, w11 = w[i00], w[i00 + dx], w[i00 + dy], w[i00 + dx + dy]
        a = w00 + fx * (w01 - w00)
        b = w10 + fx * (w11 - w10)
        r = a + fy * (b - a)
        return r - r.mean()

    def solve(self, p: SDOTProblem):
        """(weights of ``p`` in its site order, WarmStats)."""
        import torch

        with torch.cuda.stream(self._torch_stream()):
            return self._solve(p)

    def _solve(self, p: SDOTProblem):
        import torch

        t0 = time.perf_counter()
        ch = self._device_chain(p)
        chain_ms = 1e3 * (time.perf_counter() - t0)
        dev = torch.device("cuda", self.device)
        infer_ms = 0.0
        if self.start == "learned":
            from . import warmstart

            ti = time.perf_counter()
            descs = [c[0] for c in ch]
            k = self._net_level(descs)
            q = descs[k]
            # the network's inputs are host arrays of that level
            qh = SDOTProblem(f"{p.name}/level{q.n}", ch[k][1].view(-1, 2).cpu().numpy(), ch[k][2].cpu().numpy(),
                             ch[k][3].cpu().numpy(), q.size, q.proj_domain, q.grid)
            # the network through the C ABI (warmstart.CNet) or the Python host layer
            w = self.net.predict(qh) if isinstance(self.net, warmstart.CNet) else warmstart.predict(self.net, [qh])[0]
            if k != len(ch) - 1:
                qc = descs[-1]
                w = multilevel.restrict(w, qh, qc)
            w = torch.from_numpy(w).to(dev)
            infer_ms = 1e3 * (time.perf_counter() - ti)
        else:
            w = torch.zeros(ch[-1][0].n, dtype=torch.float64, device=dev)
        levels = []
        lwall = []
        dev_ms = 0.0
        for k in range(len(ch) - 1, -1, -1):
            tl = time.perf_counter()
            q, xy, nu, pic = ch[k]
            if k < len(ch) - 1:
                w = self._prolong(w, ch[k + 1][0], xy, q)
            s = self._handle(k)
            s.set_problem(xy, nu, pic, q.size, q.proj_domain)
            shrink = max(self.shrink_steps, self.shrink_coarsest if k == len(ch) - 1 else 0)
            w, st = s.solve_newton(w, tol=self.tol if k == 0 else self.coarse_tol, history=self.history,
                                   shrink_steps=shrink)
            levels.append((q.n, st))
            lwall.append(1e3 * (time.perf_counter() - tl))
            dev_ms += st.ms
        # the judge: the plain L-BFGS on the finest level's handle
        w, js = self._handle(0).solve(w, mode=capi.SOLVE_WOLFE, tol=self.tol, history=self.history,
                                      max_iter=100000)
        dev_ms += js.ms
        w = w.cpu().numpy()
        wall = 1e3 * (time.perf_counter() - t0)
        return w, WarmStats(bool(js.converged), js.max_rel_err, wall, dev_ms, infer_ms, levels, js, lwall, chain_ms)



class WarmPool:
    """Warm-started solves of many problems side by side: ``workers``
    pipelines (each a ``WarmSolver`` with its own stream and handles, kept
    between calls), each in a host thread of its own, take the problems
    round robin.  The library calls release the interpreter lock, so the
    pipelines' many small, latency-bound launches (coarse levels, Newton
    steps, the judge) overlap on the GPU instead of waiting for one another.
    Each problem's result is the one ``WarmSolver(**kw).solve`` gives (the
    same kernels on the same inputs)."""

    def __init__(self, workers: int = 4, **kw):
        self.solvers = [WarmSolver(**kw) for _ in range(max(1, int(workers)))]

    def close(self):
        for s in self.solvers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def solve_all(self, problems):
        """([(weights, WarmStats)] in problem order, wall seconds of the batch)."""
        import threading

        import torch

        workers = min(len(self.solvers), len(problems))
        out = [None] * len(problems)
        errors = []

        def run(k):
            try:
                torch.cuda.set_device(self.solvers[k].device)
                for i in range(k, len(problems), workers):
                    out[i] = self.solvers[k].solve(problems[i])
            except BaseException as e:  # reported on the calling thread
                errors.append(e)

        t0 = time.perf_counter()
        threads = [threading.Thread(target=run, args=(k,)) for k in range(workers)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
        if errors:
            raise errors[0]
        return out, wall


def solve_concurrent(problems, workers: int = 4, **kw):
    """One batch through a fresh ``WarmPool`` (its handles are set up inside
    the timed call).  Returns ([(weights, WarmStats)] in problem order, wall
    seconds)."""
    with WarmPool(workers, **kw) as pool:
        return pool.solve_all(problems)
