"""The multilevel warm start on the GPU: solves through coarse levels reach
the same tolerance as cold solves, the weights agree with the cold solve's
(the dual solution is unique up to a constant), an independent evaluation
of the returned weights confirms the error, and the finest level needs
fewer iterations than a cold solve."""
import numpy as np
import pytest

from caustic_b200 import capi, multilevel, problems

pytestmark = pytest.mark.gpu


def cold(p, tol=1e-4):
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=tol, history=10, max_iter=100000)
    s.close()
    return w, st


def max_rel(p, w):
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    _, mu, _, _ = s.eval(w)
    s.close()
    return float(np.max(np.abs(mu - p.nu) / p.nu))


@pytest.mark.parametrize("batched", [True, False])
def test_multilevel_matches_cold(gpu, batched):
    probs = [problems.make(2, 40 + i, g=64, res=512) for i in range(2)]
    ws, levels = multilevel.solve(probs, tol=1e-4, coarse_tol=1e-3, min_sites=256, batched=batched)
    assert [lv.n for lv in levels] == [256, 1024, 4096]
    assert levels[0].tol == 1e-3 and levels[-1].tol == 1e-4
    for p, w, st in zip(probs, ws, levels[-1].stats):
        assert st.converged and st.max_rel_err <= 1e-4
        assert max_rel(p, w) <= 1e-4
        wc, sc = cold(p)
        d = (w - w.mean()) - (wc - wc.mean())
        assert np.max(np.abs(d)) <= 1e-3 * np.ptp(wc)
        assert st.iterations < 0.8 * sc.iterations


def test_multilevel_start_vector(gpu):
    p = problems.make(2, 7, g=32, res=256)
    coarse = multilevel.chain(p, min_sites=256)[-1]
    w0, st0 = cold(coarse, tol=1e-3)
    ws, levels = multilevel.solve([p], w0=[w0], min_sites=256)
    # the coarsest level starts converged: a step or two at most
    assert levels[0].stats[0].iterations <= max(3, st0.iterations // 10)
    assert levels[-1].stats[0].converged and max_rel(p, ws[0]) <= 1e-4
