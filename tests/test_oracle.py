"""The CPU oracle: pinned against the reference's committed run, then checked
against independent constructions and known answers (no GPU needed)."""
import gzip
import json
import os

import numpy as np
import pytest

from caustic_b200 import problems, seeds
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _lines(name):
    with gzip.open(os.path.join(GOLD, name), "rt") as f:
        rows = f.read().splitlines()
    return [r.split() for r in rows if not r.startswith("#")]


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLD, "run.json")) as f:
        run = json.load(f)
    pts = seeds.initial_xy_point(run["point_num"], run["sample_domain"])
    proj = seeds.initial_proj_point(pts, run["sample_domain"], run["proj_domain"])
    pic = np.load(os.path.join(GOLD, "ustc_centerL.npz"))["picture"]
    dens, size = seeds.picture_from_matrix(pic)
    with gzip.open(os.path.join(GOLD, "weights0.txt.gz"), "rt") as f:
        w = np.loadtxt(f)
    return dict(run=run, pts=pts, proj=proj, dens=dens, size=size, w=w)


def test_lattice_reproduces_reference_sites(golden):
    """initial_xy_point restatement vs the reference's in.txt (6 digits)."""
    run, pts = golden["run"], golden["pts"]
    assert len(pts) == run["n_sites"] == 160978
    sub = _lines("in_sub.txt.gz")
    idx = np.array([int(a[0]) for a in sub])
    val = np.array([[float(a[1]), float(a[2])] for a in sub])
    assert np.abs(pts[idx] - val).max() < 6e-5


def test_reference_run_pins_oracle(golden):
    """At the reference's converged weights the oracle's masses and weighted
    centroids reproduce the reference run.

    The run stopped at ||mu - nu||_2 < 0.01 (configs/_py_sp_settings.json:28)
    with no empty cell; the weights were written with 6 significant digits,
    which alone moves ||mu - nu|| to ~0.08.  Without the right picture
    orientation, normalisation, source masses or centroid rule the numbers
    below are off by orders of magnitude (w = 0 gives ||g|| = 7.5)."""
    run = golden["run"]
    nu = O.source_masses(golden["pts"], run["sample_domain"])
    assert abs(nu.sum() - 1600.0) < 1e-9
    pn = O.normalize_picture(golden["dens"], run["sample_domain"])
    prob = O.Problem(golden["proj"], nu, pn, golden["size"], run["proj_domain"])
    assert list(prob.box) == [-1.0, 161.0, -61.0, 101.0]
    ev = O.evaluate(prob, golden["w"], keep_cells=True)
    g = ev.mu - nu
    assert (ev.mu == 0).sum() == 0
    assert np.linalg.norm(g) < 0.12
    g0 = O.evaluate(prob, np.zeros_like(golden["w"])).mu - nu
    assert np.linalg.norm(g0) > 50 * np.linalg.norm(g)
    c, ex = O.centers(ev.cells, pn, golden["size"], run["proj_domain"])
    assert ex.all()
    sub = _lines("out0_sub.txt.gz")
    oi = np.array([int(a[0]) for a in sub])
    ov = np.array([[float(a[1]), float(a[2])] for a in sub])
    d = np.abs(c[oi] - ov)
    assert np.median(d) < 5e-4
    assert np.percentile(d, 99) < 1e-2
    assert d.max() < 3e-2


def test_qhull_topology_matches_brute_force():
    p = problems.make(1, g=12, res=48)
    rng = np.random.default_rng(3)
    for w in (np.zeros(p.n), rng.normal(0, 0.3 / p.n, p.n)):
        a = O.cells(p.xy, w, O.proj_corner(p.xy, p.proj_domain))
        b = O.cells(p.xy, w, O.proj_corner(p.xy, p.proj_domain), brute=True)
        assert (a.ring_len == b.ring_len).all()
        assert O.adjacency(a, 1e-12) == O.adjacency(b, 1e-12)


def test_gradient_is_mass_defect_by_finite_differences():
    p = problems.make(1, g=10, res=40)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    rng = np.random.default_rng(1)
    w = rng.normal(0, 0.2 / p.n, p.n)
    d = rng.normal(0, 1.0, p.n)
    e = O.evaluate(prob, w)
    eps = 1e-8
    fd = (O.evaluate(prob, w + eps * d).f - O.evaluate(prob, w - eps * d).f) / (2 * eps)
    assert abs(fd - e.g @ d) < 1e-6 * max(1.0, abs(fd))


def test_mass_conservation_and_shift_invariance():
    p = problems.make(1, g=10, res=40)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w = np.random.default_rng(2).normal(0, 0.2 / p.n, p.n)
    e1 = O.evaluate(prob, w)
    assert abs(e1.mu.sum() - 1.0) < 1e-12
    assert abs(e1.g.sum()) < 1e-12
    e2 = O.evaluate(prob, w + 0.37)
    assert np.abs(e1.mu - e2.mu).max() < 1e-12


def test_uniform_density_square_lattice_is_balanced_at_zero():
    """Known answer: equal cells on a square lattice with uniform density."""
    g = 8
    a = (np.arange(g) + 0.5) / g
    X, Y = np.meshgrid(a, a)
    xy = np.stack([X.ravel(), Y.ravel()], 1)
    nu = np.full(g * g, 1.0 / (g * g))
    prob = O.Problem(xy, nu, np.full(32 * 32, 1.0 / 1024), (32, 32), problems.UNIT_DOMAIN)
    e = O.evaluate(prob, np.zeros(g * g))
    assert np.abs(e.mu - nu).max() < 1e-14


def test_two_sites_split_line():
    """Known answer: two sites, bisector moved by the weight difference."""
    xy = np.array([[0.25, 0.5], [0.75, 0.5]])
    nu = np.array([0.5, 0.5])
    prob = O.Problem(xy, nu, np.full(16, 1 / 16.0), (4, 4), problems.UNIT_DOMAIN)
    for dw in (0.0, 0.1, -0.05):
        # |x-s0|^2 - w0 = |x-s1|^2 - w1  ->  x = 0.5 + (w0 - w1) / (2 * 0.5)
        xs = 0.5 + dw / 1.0
        e = O.evaluate(prob, np.array([dw, 0.0]))
        assert abs(e.mu[0] - xs) < 1e-14
        assert abs(e.mu[1] - (1 - xs)) < 1e-14


def test_hidden_cell_has_no_mass():
    p = problems.make(1, g=6, res=24)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w = np.zeros(p.n)
    w[14] = -1.0          # far below its neighbours: the cell vanishes
    e = O.evaluate(prob, w, keep_cells=True)
    assert e.mu[14] == 0.0 and e.cells.ring_len[14] == 0
    assert abs(e.fcell[14] - (-w[14] * p.nu[14])) < 1e-15


def test_reference_solver_restatement_converges():
    p = problems.make(1, g=8, res=32)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = O.direct_ot_parity(prob, np.zeros(p.n), total_iter=500, tol=1e-5, m=7)
    assert st.converged
    e = O.evaluate(prob, w)
    assert np.linalg.norm(e.g) < 1e-5 + 1e-7
    assert abs(w.sum()) < 1e-9   # sum(g) = 0 keeps sum(w) at its start value


def test_wolfe_solver_reaches_max_relative_tolerance():
    p = problems.make(1, g=8, res=32)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = O.lbfgs_wolfe(prob, np.zeros(p.n), tol=1e-4)
    assert st.converged
    assert O.max_rel_error(O.evaluate(prob, w).mu, p.nu) <= 1e-4


def test_wolfe_solver_passes_the_evaluation_noise_floor(monkeypatch):
    """Near convergence the objective's evaluation noise exceeds what a step
    can still gain; with the approximate Wolfe rule the solve goes on to
    1e-10, without it (F_NOISE = 0) it stalls after 50 failed searches."""
    p = problems.make(2, 0, g=8, res=32)
    prob = O.Problem(p.xy, p.nu, p.picture, np.array(p.size), p.proj_domain)
    w, st = O.lbfgs_wolfe(prob, np.zeros(p.n), tol=1e-10, max_iter=3000)
    assert st.converged and st.restarts == 0
    assert O.max_rel_error(O.evaluate(prob, w).mu, p.nu) <= 1e-10
    monkeypatch.setattr(O, "F_NOISE", 0.0)
    _, st0 = O.lbfgs_wolfe(prob, np.zeros(p.n), tol=1e-10, max_iter=3000)
    assert not st0.converged and st0.restarts > 50


def test_green_integral_is_exact_second_moment():
    """Polygon_Ints (basic_function.cuh:826-865) = int |x - s|^2 for CCW rings."""
    L = O.lib()
    sq = np.array([1.0, 2.0, 3.0, 2.0, 3.0, 5.0, 1.0, 5.0])
    s = np.array([0.3, -0.7])
    # int over [1,3]x[2,5] of (x-sx)^2 + (y-sy)^2
    ix = ((3 - s[0]) ** 3 - (1 - s[0]) ** 3) / 3 * 3
    iy = ((5 - s[1]) ** 3 - (2 - s[1]) ** 3) / 3 * 2
    v = L.orc_poly_ints(O._d(sq), 4, O._d(s))
    assert abs(v - (ix + iy)) < 1e-12 * abs(ix + iy)


def test_mass_jacobian_by_finite_differences():
    """The masses' Jacobian (edge density integrals over 2|s_i - s_j|, the
    Newton solve's matrix) against central differences of the masses."""
    p = problems.make(1, g=12, res=48, beam=True)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    rng = np.random.default_rng(4)
    w = rng.normal(0, 0.3 / p.n, p.n)
    J = O.mass_jacobian(prob, w)
    assert abs(J - J.T).max() < 1e-12 * abs(J).max()           # symmetric
    assert np.abs(np.asarray(J.sum(axis=1))).max() < 1e-12 * abs(J).max()   # rows sum to zero
    for _ in range(3):
        d = rng.normal(0, 1.0 / p.n, p.n)
        eps = 1e-4
        fd = (O.evaluate(prob, w + eps * d).mu - O.evaluate(prob, w - eps * d).mu) / (2 * eps)
        assert np.abs(fd - J @ d).max() < 1e-5 * np.abs(fd).max()


def test_mass_jacobian_known_answer():
    """Two sites on a uniform density: the shared edge is the vertical line
    x = 0.5 + (w0 - w1) of length 1, and |s0 - s1| = 0.5, so
    dmu0/dw1 = -1 / (2 * 0.5) = -1."""
    xy = np.array([[0.25, 0.5], [0.75, 0.5]])
    prob = O.Problem(xy, np.array([0.5, 0.5]), np.full(16, 1 / 16.0), (4, 4), problems.UNIT_DOMAIN)
    J = O.mass_jacobian(prob, np.array([0.05, 0.0])).toarray()
    assert np.allclose(J, [[1.0, -1.0], [-1.0, 1.0]], atol=1e-14)
