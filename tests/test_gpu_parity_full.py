"""GPU path against the CPU oracle at the benchmark sizes.

The timed workload (N = 65,536 sites, 1024^2 image, beam masses) is checked
in full: masses and gradients within 1e-10 of the largest mass, the
objective within 1e-9 of the sum of |f_i|, and cell adjacency bit-exact for
every shared edge longer than 1e-9 of the site pitch -- at w = 0, at the
iterate after 200 L-BFGS iterations and at the converged weights.  The
largest instance of the batched configuration (N = 32,041, 512^2) and one
evaluation at the combined configuration's size (N = 262,144, 2048^2) take
the same checks.  The path replaced is the reference's per-cell integration
(Optimal_Transport_rl/basic_function.cuh:743-952) over CGAL's power cells
(power_diagram.cpp:8-134).
"""
import numpy as np
import pytest

from caustic_b200 import capi, problems
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MU_TOL = 1e-10
F_TOL = 1e-9


def edge_pairs(off, xy, nb, min_len):
    """Set-free adjacency: sorted unique (i, j) rows, i < j, for ring edges
    whose neighbour is a site and whose length exceeds min_len."""
    off = np.asarray(off, np.int64)
    n = len(off) - 1
    lens = np.diff(off)
    owner = np.repeat(np.arange(n), lens)
    nxt = np.arange(len(nb)) + 1
    last = off[1:] - 1
    nxt[last[lens > 0]] = off[:-1][lens > 0]
    ln = np.hypot(*(xy[nxt] - xy).T)
    keep = (nb >= 0) & (ln > min_len)
    a, b = owner[keep], nb[keep].astype(np.int64)
    pairs = np.stack([np.minimum(a, b), np.maximum(a, b)], axis=1)
    return np.unique(pairs, axis=0)


def oracle_pairs(c: O.Cells, min_len):
    lens = c.lens()
    n = len(lens)
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(lens)
    xy = np.concatenate([c.ring_xy[i, :lens[i]] for i in range(n) if lens[i] > 0])
    nb = np.concatenate([c.ring_lab[i, :lens[i]] for i in range(n) if lens[i] > 0])
    return edge_pairs(off, xy, nb, min_len)


def check_full(p, s, w, cap=256):
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain, cap=cap)
    f, mu, g, fc = s.eval(w)
    ev = O.evaluate(prob, w, keep_cells=True)
    assert (ev.cells.ring_len >= 0).all(), "a ring above the oracle's capacity"
    scale = np.abs(ev.mu).max()
    assert np.abs(mu - ev.mu).max() <= MU_TOL * scale
    assert np.abs(g - ev.g).max() <= MU_TOL * scale
    assert abs(f - ev.f) <= F_TOL * max(abs(ev.f), np.abs(ev.fcell).sum())
    pd = p.proj_domain
    pitch = np.sqrt((pd[1] - pd[0]) * (pd[3] - pd[2]) / p.n)
    off, gxy, gnb = s.cells(w)
    ga = edge_pairs(off, gxy, gnb, 1e-9 * pitch)
    oa = oracle_pairs(ev.cells, 1e-9 * pitch)
    assert ga.shape == oa.shape and np.array_equal(ga, oa)
    return ev


def test_config2_full_size_parity(gpu):
    """The benchmark workload, N = 65,536 and 1024^2: at the cold start, in
    the middle of the solve (after 200 iterations, where cells of the 1e-3
    floor are large and many are still hidden) and at the solution."""
    p = problems.make(2)
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    check_full(p, s, np.zeros(p.n))
    w200, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10, max_iter=200)
    assert st.iterations == 200 and not st.converged
    ev = check_full(p, s, w200)
    assert (ev.mu == 0).sum() > 0 or O.max_rel_error(ev.mu, p.nu) > 1e-2   # a genuinely mid-solve point
    wsol, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    assert st.converged
    ev = check_full(p, s, wsol)
    assert O.max_rel_error(ev.mu, p.nu) <= 1e-4 * (1 + 1e-6)


def test_config3_largest_instance_parity(gpu):
    """The largest of the 64 batched instances (N = 32,041, 512^2, uniform
    masses) at w = 0 and after 150 iterations."""
    p = max((problems.make(3, i) for i in range(64)), key=lambda q: q.n)
    assert p.n == 32041
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    check_full(p, s, np.zeros(p.n))
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10, max_iter=150)
    check_full(p, s, w)


def test_config5_size_evaluation_parity(gpu):
    """One instance of the combined configuration's size (N = 262,144,
    2048^2, beam masses): w = 0 and a random weight field of the size that
    hides cells."""
    p = problems.make(5)
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    check_full(p, s, np.zeros(p.n), cap=64)
    w = np.random.default_rng(55).normal(0.0, 0.5 / p.n, p.n)
    ev = check_full(p, s, w, cap=64)
    assert (ev.mu == 0).sum() > 0
