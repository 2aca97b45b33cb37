"""The warm-start pipeline (caustic_b200/warm.py) on the GPU: multilevel
damped Newton levels, then the plain L-BFGS as the judge.  The result is
judged again by the oracle, and it is the cold solve's solution (the dual
solution is unique up to a constant)."""
import os

import numpy as np
import pytest

from caustic_b200 import capi, problems, warmstart
from caustic_b200.warm import WarmSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NET = os.path.join(os.path.dirname(warmstart.__file__), "data", "warmstart_c2_64.npz")   # trained at 64^2 sites


def oracle_err(p, w):
    return O.max_rel_error(O.evaluate(O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain), w).mu, p.nu)


def test_multilevel_newton_pipeline(gpu):
    p = problems.make(2, 11, g=64, res=256)
    with WarmSolver(start="multilevel", min_sites=256) as ws:
        w, st = ws.solve(p)
        w2, st2 = ws.solve(p)          # the same handles again: the same bits
    assert st.converged and st.max_rel_err <= 1e-4
    assert [n for n, _ in st.levels] == [256, 1024, 4096]
    assert all(not x.fallback for _, x in st.levels)
    assert st.judge.iterations == 0 and st.judge.evaluations == 1   # the judge confirms at once
    assert np.array_equal(w, w2)
    assert oracle_err(p, w) <= 1e-4 * (1 + 1e-6)
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    wc, sc = s.solve(np.zeros(p.n), tol=1e-6)
    assert np.abs((w - w.mean()) - (wc - wc.mean())).max() < 1e-3 * np.ptp(wc)
    # the whole pipeline costs a fraction of the cold solve's evaluations
    evals = sum(x.evaluations for _, x in st.levels) + st.judge.evaluations
    assert evals < 0.2 * sc.evaluations


@pytest.mark.skipif(not os.path.exists(NET), reason="no trained network in the package")
def test_learned_start_saves_damped_steps(gpu):
    """The trained network's prediction, averaged down to the coarsest level,
    starts that level closer to its solution than w = 0: fewer damped Newton
    steps there, the same finest tolerance at the end, judged by the plain
    L-BFGS and the oracle."""
    p = problems.make(2, 7)
    net = warmstart.WarmStartNet.from_file(NET)
    with WarmSolver(start="multilevel") as ml, WarmSolver(start="learned", net=net, net_level_sites=4096) as le:
        _, sm = ml.solve(p)
        w, sl = le.solve(p)
    assert sm.converged and sl.converged
    assert [n for n, _ in sl.levels] == [n for n, _ in sm.levels]
    assert sl.levels[0][1].newton_iterations < sm.levels[0][1].newton_iterations
    assert oracle_err(p, w) <= 1e-4 * (1 + 1e-6)


def test_concurrent_pipelines_match_sequential(gpu):
    """Four problems warm-solved by two pipelines side by side (host threads,
    one stream each) give the weights of one pipeline solving them in turn,
    bit for bit, every one converged."""
    from caustic_b200.warm import solve_concurrent

    ps = [problems.make(2, 20 + i, g=64, res=256) for i in range(4)]
    with WarmSolver(start="multilevel", min_sites=256) as ws:
        seq = [ws.solve(p) for p in ps]
    con, wall = solve_concurrent(ps, workers=2, start="multilevel", min_sites=256)
    assert wall > 0
    for (w1, s1), (w2, s2) in zip(seq, con):
        assert s1.converged and s2.converged and s2.max_rel_err <= 1e-4
        assert np.array_equal(w1, w2)
