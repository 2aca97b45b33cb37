"""Restriction and prolongation of the multilevel warm start (host code,
no GPU): merged sites keep the total mass and the image its total, the
image is merged only while it stays fine against the coarse sites, and the
prolongation reproduces a linear function of the position inside the
lattice."""
import numpy as np
import pytest

from caustic_b200 import multilevel, problems


def test_coarsen_keeps_masses_and_image():
    p = problems.make(2, 3, g=32, res=256)
    c = multilevel.coarsen(p)
    assert c.grid == (16, 16) and c.n == 256
    assert c.nu.sum() == pytest.approx(p.nu.sum(), rel=1e-14)
    # 256 px over 16 coarse sites: 16 per site, so the image is merged too
    assert c.size == (128, 128)
    assert c.picture.sum() == pytest.approx(np.sum(p.picture), rel=1e-14)
    # each coarse site is the mean of its 2 x 2 block
    blk = p.xy.reshape(16, 2, 16, 2, 2)[3, :, 5, :, :].reshape(4, 2).mean(axis=0)
    assert np.allclose(c.xy[3 * 16 + 5], blk)


def test_coarse_image_kept_when_too_close_to_the_pitch():
    p = problems.make(4, 0, g=32, res=64)
    c = multilevel.coarsen(p)           # 64 px over 16 coarse sites: 4 each
    assert c.size == (64, 64)
    np.testing.assert_array_equal(c.picture, p.picture)
    c2 = multilevel.coarsen(c)          # 64 px over 8: 8 each, merged
    assert c2.size == (32, 32)


def test_chain_depth_and_odd_lattices():
    p = problems.make(2, 0, g=64, res=512)
    ch = multilevel.chain(p, min_sites=256)
    assert [q.grid for q in ch] == [(64, 64), (32, 32), (16, 16)]
    odd = problems.make(1, 0, g=6, res=32)
    assert len(multilevel.chain(odd, min_sites=4)) == 2  # 6 -> 3, then odd
    with pytest.raises(ValueError):
        multilevel.coarsen(multilevel.coarsen(odd))


def test_prolong_reproduces_linear_functions_inside():
    p = problems.make(2, 1, g=32, res=128)
    c = multilevel.coarsen(p)
    gx, gy = c.grid
    a, b = np.meshgrid(np.arange(gx), np.arange(gy))
    lattice = np.stack([(a.ravel() + 0.5) / gx, (b.ravel() + 0.5) / gy], axis=1)

    def f(q):
        return 3.0 * q[:, 0] - 2.0 * q[:, 1]

    w = multilevel.prolong(f(lattice), c, p)
    assert abs(w.mean()) < 1e-12
    inside = ((p.xy[:, 0] > 0.5 / gx) & (p.xy[:, 0] < 1 - 0.5 / gx) &
              (p.xy[:, 1] > 0.5 / gy) & (p.xy[:, 1] < 1 - 0.5 / gy))
    d = (w - f(p.xy))[inside]           # a constant: the removed mean
    assert np.ptp(d) < 1e-12


def test_multilevel_chain_with_the_oracle_as_level_solver():
    """The whole chain on the CPU, each level solved by the oracle's Wolfe
    L-BFGS: the finest level reaches the tolerance and needs fewer
    iterations than a cold solve of the same problem."""
    from types import SimpleNamespace

    from oracle import oracle as O

    def oprob(q):
        return O.Problem(q.xy, q.nu, q.picture, np.array(q.size), q.proj_domain)

    def level_solver(level, starts, tol):
        ws, st = [], []
        for q, w in zip(level, starts):
            w, s = O.lbfgs_wolfe(oprob(q), w, tol=tol)
            err = O.max_rel_error(O.evaluate(oprob(q), w).mu, q.nu)
            ws.append(w)
            st.append(SimpleNamespace(iterations=s.iterations, max_rel_err=err, converged=s.converged))
        return ws, st, 0.0

    p = problems.make(2, 3, g=32, res=256)
    ws, levels = multilevel.solve([p], min_sites=64, level_solver=level_solver)
    assert [lv.n for lv in levels] == [64, 256, 1024]
    assert [lv.tol for lv in levels] == [1e-3, 1e-3, 1e-4]
    fine = levels[-1].stats[0]
    assert fine.converged and fine.max_rel_err <= 1e-4
    _, cold = O.lbfgs_wolfe(oprob(p), np.zeros(p.n), tol=1e-4)
    assert fine.iterations < 0.8 * cold.iterations
