"""Batched solves (cot_solve_batch): one graph launch, one branch per
instance.  Batching changes nothing in any instance's arithmetic, so every
batched solve is bit-identical to the same solve on its own."""
import numpy as np
import pytest

from caustic_b200 import batch, capi, problems

pytestmark = pytest.mark.gpu


def uneven():
    return [problems.make(1, instance=i, g=g, res=64, beam=bool(i % 2)) for i, g in enumerate((8, 31, 12, 20, 16, 27))]


def solvers_for(probs, **kw):
    out = []
    for p in probs:
        s = capi.Solver(**kw)
        s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        out.append(s)
    return out


@pytest.mark.parametrize("mode", [capi.SOLVE_WOLFE, capi.SOLVE_REFERENCE])
def test_batch_matches_single_solves(gpu, mode):
    probs = uneven()
    tol = 1e-4 if mode == capi.SOLVE_WOLFE else 1e-5
    sol = solvers_for(probs)
    wb, sb = capi.solve_batch(sol, [np.zeros(p.n) for p in probs], mode=mode, tol=tol, history=7, max_iter=3000)
    for k, (p, s) in enumerate(zip(probs, sol)):
        one = capi.Solver()
        one.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        w1, s1 = one.solve(np.zeros(p.n), mode=mode, tol=tol, history=7, max_iter=3000)
        assert sb[k].converged and s1.converged
        assert (sb[k].iterations, sb[k].evaluations) == (s1.iterations, s1.evaluations)
        assert np.array_equal(wb[k], w1)
        assert s.kernel_stats()["evaluations"] == one.kernel_stats()["evaluations"]
    assert len({x.ms for x in sb}) == 1   # one time for the whole batch


def test_batch_stops_and_reports(gpu):
    probs = uneven()[:3]
    sol = solvers_for(probs)
    wb, sb = capi.solve_batch(sol, [np.zeros(p.n) for p in probs], tol=1e-12, max_iter=25)
    assert all(x.iterations == 25 and not x.converged for x in sb)
    with pytest.raises(capi.CotError) as e:
        capi.solve_batch(sol, [np.zeros(p.n) for p in probs], tol=1e-12, max_iter=25, raise_on_noconv=True)
    assert e.value.code == capi.COT_ENOTCONV
    with pytest.raises(capi.CotError) as e:
        capi.solve_batch([sol[0], sol[1], sol[0]], [np.zeros(p.n) for p in (probs[0], probs[1], probs[0])])
    assert e.value.code == capi.COT_EINVAL
    with pytest.raises(ValueError):
        capi.solve_batch(sol, [np.zeros(3)] * 3)


def test_autotune_and_batched_config_instances(gpu):
    probs = batch.instances(6, res=64)
    assert len({p.n for p in probs}) > 3 and all(1024 * 0.9 <= p.n <= 32768 * 1.1 for p in probs)
    res = batch.autotune(probs, sample=3, max_iter=8, bucket_sizes=(8, 16))
    assert len(res.table) == len(batch.CELLS_PER_WARP) * 2
    assert (res.cells_per_warp, res.bucket_size) in [(c, b) for c, b, _ in res.table]
    ws, st, sec = batch.solve(probs[:3], cells_per_warp=res.cells_per_warp, bucket_size=res.bucket_size,
                              max_iter=40)
    assert sec > 0 and all(x.iterations <= 40 for x in st)
