"""Progress reports during a solve (cot_set_progress): the schedule, the
phase sequence of aarl_direct_ot, cancellation, and that queries made from
inside the callback leave the solve untouched."""
import numpy as np
import pytest

from caustic_b200 import capi, problems

pytestmark = pytest.mark.gpu


def solver_for(p):
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    return s


def test_schedule_and_final_report(gpu):
    p = problems.make(1, g=16, res=64)
    s = solver_for(p)
    seen = []
    s.set_progress(lambda ph, it, st, w, nu, g, m: seen.append((ph, it, st, w, nu, g, m)), every=10)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_REFERENCE, tol=1e-5, history=7, max_iter=2000)
    assert st.converged
    its = [x[1] for x in seen]
    assert its[0] == -1 and seen[0][2] == 0
    assert all(x[0] == capi.PHASE_LBFGS for x in seen)
    assert its[1:-1] == list(range(0, st.iterations - 1, 10))
    last = seen[-1]
    assert last[1] == st.iterations - 1 and last[2] == 1
    assert np.array_equal(last[3], w)
    assert np.array_equal(seen[0][4], p.nu)      # the problem's masses in caller order
    assert np.allclose(seen[0][3], 0.0)


def test_queries_inside_the_callback_leave_the_solve_alone(gpu):
    """Renders and evaluations from the callback use their own weight
    buffer: the solve's trajectory is bit-identical with and without them."""
    p = problems.make(1, g=16, res=64, beam=True)
    a = solver_for(p)
    w_plain, st_plain = a.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    b = solver_for(p)
    imgs = []

    def cb(ph, it, st, w, nu, g, m):
        imgs.append(b.render(w, 1.0).sum())
        b.eval(np.full(p.n, 0.3 / p.n))          # an unrelated point
        b.centroids(w)
        return False

    b.set_progress(cb, every=7)
    w_cb, st_cb = b.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    assert len(imgs) > 3
    assert st_cb.iterations == st_plain.iterations and st_cb.evaluations == st_plain.evaluations
    assert np.array_equal(w_cb, w_plain)


def test_callback_stops_the_solve(gpu):
    p = problems.make(1, g=16, res=64)
    s = solver_for(p)
    got = {}

    def cb(ph, it, st, w, nu, g, m):
        got[it] = w
        return it >= 20

    s.set_progress(cb, every=5)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-12, history=10)
    assert not st.converged and st.iterations == 21
    assert np.array_equal(w, got[20])
    with pytest.raises(capi.CotError) as e:
        s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-12, history=10, raise_on_noconv=True)
    assert e.value.code == capi.COT_ECANCELLED
    # an exception in the callback stops the solve and comes back out of it
    def bad(ph, it, st, w, nu, g, m):
        raise KeyError("from the callback")

    s.set_progress(bad)
    with pytest.raises(KeyError):
        s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-12, history=10)
    s.set_progress(None)
    _, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    assert st.converged


def test_aarl_phase_sequence(gpu):
    p = problems.make(1, g=12, res=48)
    rng = np.random.default_rng(5)
    n = p.n
    pts = p.xy * 40.0
    inl = np.tile([0.0, 0.0, 1.0], (n, 1))
    insl = np.column_stack([rng.normal(0, 0.05, n), rng.normal(0, 0.05, n), np.ones(n)])
    insl /= np.linalg.norm(insl, axis=1, keepdims=True)
    hgt = rng.uniform(5, 10, n)
    kw = dict(z_of_len=0.0, z_of_receiver=3.0, refraction_index=1.5, sample_domain=[0, 40, 0, 40], aa_history=7,
              aa_fixed_para=-0.3, history=7, max_iter=300, tol=3e-6)
    s = solver_for(p)
    seen = []
    s.set_progress(lambda ph, it, st, w, nu, g, m: seen.append((ph, it, st, nu)), every=25)
    w, st = s.solve_aarl(np.zeros(n), pts, inl, insl, hgt, lbfgs_prepass=True, **kw)
    assert st.converged
    phases = [x[0] for x in seen]
    k = phases.index(capi.PHASE_ANDERSON)
    assert seen[0][:2] == (capi.PHASE_PREPASS, -1)
    assert all(ph == capi.PHASE_PREPASS for ph in phases[:k]) and all(ph == capi.PHASE_ANDERSON for ph in phases[k:])
    assert seen[k - 1][2] in (1, 2)                 # the pre-pass ended
    assert seen[k][1] == -1 and seen[-1][2] == 1
    assert abs(seen[0][3].sum() - p.nu.sum()) < 1e-12   # re-weighted masses keep the total
    assert not np.array_equal(seen[0][3], p.nu)
    # the same solve without the callback
    t = solver_for(p)
    w2, st2 = t.solve_aarl(np.zeros(n), pts, inl, insl, hgt, lbfgs_prepass=True, **kw)
    assert st2.iterations == st.iterations and np.array_equal(w, w2)
    # without the pre-pass the pre-pass phase still reports its start
    u = solver_for(p)
    seen2 = []
    u.set_progress(lambda ph, it, st, w, nu, g, m: seen2.append((ph, it)), every=1000)
    u.solve_aarl(np.zeros(n), pts, inl, insl, hgt, lbfgs_prepass=False, **dict(kw, max_iter=30, tol=1e-12))
    assert seen2[0] == (capi.PHASE_PREPASS, -1) and seen2[1] == (capi.PHASE_ANDERSON, -1)
    assert seen2[-1] == (capi.PHASE_ANDERSON, 29)
