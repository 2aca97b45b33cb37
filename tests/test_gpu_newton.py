"""The damped Newton solve (cot_solve_newton) and its Jacobian
(cot_mass_jacobian) against the CPU oracle.

The Jacobian dmu/dw has no counterpart in the reference; its oracle is
oracle.mass_jacobian (edge density integrals over 2|s_i - s_j|), itself
checked against finite differences of the oracle's masses.  The solve's
result is judged as the L-BFGS's is: the oracle's masses at the returned
weights are within the tolerance of the targets.
"""
import numpy as np
import pytest

from caustic_b200 import capi, problems
from oracle import oracle as O

pytestmark = pytest.mark.gpu

J_TOL = 1e-9   # relative to the largest entry: edge integrals summed in another order


def oracle_problem(p):
    return O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)


def solver_for(p, **kw):
    s = capi.Solver(**kw)
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    return s


@pytest.mark.parametrize("g,res,scale", [(24, 96, 0.3), (32, 128, 1.0)])
def test_jacobian_matches_oracle(gpu, g, res, scale):
    p = problems.make(1, g=g, res=res, beam=True)
    s = solver_for(p)
    w = np.random.default_rng(g).normal(0.0, scale / p.n, p.n)
    J = s.mass_jacobian(w).toarray()
    R = O.mass_jacobian(oracle_problem(p), w).toarray()
    assert np.abs(J - R).max() <= J_TOL * np.abs(R).max()
    # rows sum to zero: moving every weight together moves no edge
    assert np.abs(J.sum(axis=1)).max() <= 1e-12 * np.abs(R).max()
    # and the GPU's own masses move as the Jacobian says
    d = np.random.default_rng(1).normal(0.0, 1.0 / p.n, p.n)
    eps = 1e-4
    fd = (s.eval(w + eps * d)[1] - s.eval(w - eps * d)[1]) / (2 * eps)
    assert np.abs(fd - J @ d).max() <= 1e-5 * np.abs(fd).max()


def test_jacobian_with_long_rings(gpu):
    """Heavy sites make rings above 32 vertices: their rows come from the
    large-ring pass."""
    p = problems.make(1, g=32, res=128, beam=True)
    rng = np.random.default_rng(23)
    w = rng.normal(0, 0.3 / p.n, p.n)
    order = np.argsort(p.xy[:, 0] * 7 + p.xy[:, 1])
    heavy = order[[150, 500, 850, 300, 700]]
    w[heavy[:3]] += 15.0 / p.n
    w[heavy[3:]] += 40.0 / p.n
    s = solver_for(p)
    off, _, _ = s.cells(w)
    assert (np.diff(off) > 32).sum() >= 2
    J = s.mass_jacobian(w).toarray()
    R = O.mass_jacobian(oracle_problem(p), w).toarray()
    assert np.abs(J - R).max() <= J_TOL * np.abs(R).max()


def test_newton_solve_small(gpu):
    p = problems.make(1, g=32, res=128, beam=True)
    s = solver_for(p)
    w, st = s.solve_newton(np.zeros(p.n), tol=1e-4)
    assert st.converged and not st.fallback and st.newton_iterations > 0
    assert O.max_rel_error(O.evaluate(oracle_problem(p), w).mu, p.nu) <= 1e-4 * (1 + 1e-6)
    # the same solution as the L-BFGS's (weights up to a constant)
    wl, sl = solver_for(p).solve(np.zeros(p.n), tol=1e-6)
    span = np.ptp(wl)
    assert np.abs((w - w.mean()) - (wl - wl.mean())).max() < 1e-2 * span
    # bit for bit again, on a fresh handle and on the same one
    w2, st2 = solver_for(p).solve_newton(np.zeros(p.n), tol=1e-4)
    assert np.array_equal(w, w2) and st2.cg_iterations == st.cg_iterations
    w3, _ = s.solve_newton(np.zeros(p.n), tol=1e-4)
    assert np.array_equal(w, w3)


def test_newton_solve_tight_tolerance(gpu):
    """Newton steps converge quadratically near the solution: 1e-9 in a few
    more steps than 1e-4."""
    p = problems.make(2, 0, g=16, res=64)
    s = solver_for(p)
    w4, st4 = s.solve_newton(np.zeros(p.n), tol=1e-4)
    w9, st9 = s.solve_newton(np.zeros(p.n), tol=1e-9)
    assert st9.converged and not st9.fallback
    assert st9.newton_iterations <= st4.newton_iterations + 6
    assert O.max_rel_error(O.evaluate(oracle_problem(p), w9).mu, p.nu) <= 1e-8


def test_newton_config2_full_size(gpu):
    """The benchmark workload from the cold start, judged by the oracle."""
    p = problems.make(2)
    s = solver_for(p)
    w, st = s.solve_newton(np.zeros(p.n), tol=1e-4)
    assert st.converged, st
    assert O.max_rel_error(O.evaluate(oracle_problem(p), w).mu, p.nu) <= 1e-4 * (1 + 1e-6)


def test_set_problem_reuses_buffers(gpu):
    """A smaller problem on the same handle reuses its buffers (and the
    Newton buffers and history sized for the larger one); a larger one
    reallocates.  Results are the same as on fresh handles."""
    big = problems.make(1, g=32, res=128, beam=True)
    small = problems.make(1, 3, g=20, res=80)
    s = capi.Solver()
    for p in (big, small, big):
        s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        w, st = s.solve(np.zeros(p.n), tol=1e-4)
        wf, stf = solver_for(p).solve(np.zeros(p.n), tol=1e-4)
        assert st.converged and np.array_equal(w, wf) and st.evaluations == stf.evaluations
        wn, sn = s.solve_newton(np.zeros(p.n), tol=1e-4)
        wnf, _ = solver_for(p).solve_newton(np.zeros(p.n), tol=1e-4)
        assert sn.converged and np.array_equal(wn, wnf)
