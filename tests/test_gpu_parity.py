"""GPU path (libcausticot.so through the C ABI) against the CPU oracle.

Tolerances: cell masses and gradients agree to 1e-10 relative to the largest
mass; the objective to 1e-9 relative (it is a sum of terms of both signs);
adjacency bit-exact for every shared edge longer than 1e-9 of the site pitch.
"""
import gzip
import json
import os

import numpy as np
import pytest

from caustic_b200 import capi, problems, seeds
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

MU_TOL = 1e-10
F_TOL = 1e-9


def oracle_problem(p):
    return O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)


def solver_for(p, **kw):
    s = capi.Solver(**kw)
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    return s


def gpu_adjacency(s, w, min_len):
    off, xy, nb = s.cells(w)
    out = set()
    for i in range(len(off) - 1):
        R = xy[off[i]:off[i + 1]]
        L = nb[off[i]:off[i + 1]]
        if len(R) == 0:
            continue
        Q = np.roll(R, -1, axis=0)
        ln = np.hypot(*(Q - R).T)
        for k in range(len(L)):
            if L[k] >= 0 and ln[k] > min_len:
                out.add((min(i, int(L[k])), max(i, int(L[k]))))
    return out, off


def check_eval(p, w, s=None):
    prob = oracle_problem(p)
    s = s or solver_for(p)
    f, mu, g, fc = s.eval(w)
    ev = O.evaluate(prob, w, keep_cells=True)
    scale = np.abs(ev.mu).max()
    assert np.abs(mu - ev.mu).max() <= MU_TOL * scale
    assert np.abs(g - ev.g).max() <= MU_TOL * scale
    assert abs(f - ev.f) <= F_TOL * max(abs(ev.f), np.abs(ev.fcell).sum())
    pd = p.proj_domain
    pitch = np.sqrt((pd[1] - pd[0]) * (pd[3] - pd[2]) / p.n)
    ga, _ = gpu_adjacency(s, w, 1e-9 * pitch)
    oa = O.adjacency(ev.cells, 1e-9 * pitch)
    assert ga == oa
    return s, ev


@pytest.mark.parametrize("g,res,beam", [(8, 32, False), (24, 96, False), (32, 128, True)])
def test_eval_parity_small(gpu, g, res, beam):
    p = problems.make(1, g=g, res=res, beam=beam)
    s = solver_for(p)
    rng = np.random.default_rng(g)
    check_eval(p, np.zeros(p.n), s)
    check_eval(p, rng.normal(0, 0.3 / p.n, p.n), s)
    check_eval(p, rng.normal(0, 1.0 / p.n, p.n), s)   # strongly weighted: hidden cells appear


def test_eval_parity_config1_full(gpu):
    """N=4096, 256x256 mixture: masses, gradient, objective, adjacency."""
    p = problems.make(1)
    s = solver_for(p)
    check_eval(p, np.zeros(p.n), s)
    w = np.random.default_rng(11).normal(0, 0.5 / p.n, p.n)
    check_eval(p, w, s)


@pytest.mark.parametrize("nx,ny,pd", [
    (160, 160, [0.0, 1.0, 0.0, 1.0]),
    (97, 131, [0.0, 16.0, -6.0, 10.0]),
    (333, 45, [-3.3, 7.1, 0.7, 2.9]),
    (7, 5, [0.1, 0.9, 0.2, 0.8]),
    (1, 1, [-1.0, 1.0, -1.0, 1.0]),
])
def test_eval_parity_across_grids(gpu, nx, ny, pd):
    """Odd, non-square and offset pixel grids: a cell edge on the domain's
    far sides sits where the pixel lines computed from the grid origin and
    step may round either way of it."""
    rng = np.random.default_rng(nx * 1000 + ny)
    gx, gy = 23, 17
    u = (np.arange(gx) + 0.5 + rng.uniform(-0.3, 0.3, (gy, gx))) / gx
    v = ((np.arange(gy) + 0.5)[:, None] + rng.uniform(-0.3, 0.3, (gy, gx))) / gy
    xy = np.column_stack([pd[0] + (pd[1] - pd[0]) * u.ravel(), pd[2] + (pd[3] - pd[2]) * v.ravel()])
    n = len(xy)
    nu = rng.uniform(0.5, 1.5, n)
    nu /= nu.sum()
    pic = rng.uniform(0.0, 1.0, nx * ny) ** 2
    pic[rng.uniform(size=nx * ny) < 0.1] = 0.0
    pic /= pic.sum()
    p = problems.SDOTProblem("grid", xy, nu, pic, (nx, ny), np.array(pd, float))
    s = solver_for(p)
    scale = ((pd[1] - pd[0]) * (pd[3] - pd[2])) / n
    for w in (np.zeros(n), rng.normal(0, 0.5 * scale, n)):
        check_eval(p, w, s)
        c = O.cells(p.xy, w, O.proj_corner(p.xy, p.proj_domain))
        xyc, ex = s.centroids(w, weighted=True)
        oxy, oex = O.centers(c, p.picture, p.size, p.proj_domain, weighting=True)
        assert np.array_equal(ex, oex)
        assert np.abs(xyc[ex] - oxy[ex]).max() < 1e-10 * max(pd[1] - pd[0], pd[3] - pd[2])


@pytest.mark.parametrize("bucket", [1, 2, 5, 16, 64, 100000])
def test_eval_parity_across_bucket_sizes(gpu, bucket):
    """The bucket grid only changes which candidates are tried first and how
    the bound tree is shaped (1-2 sites per bucket overflows the traversal
    frontier and takes the every-bucket scan; one bucket for everything
    leaves a single leaf): masses and adjacency stay the oracle's."""
    p = problems.make(1, g=40, res=160, beam=True)
    s = solver_for(p, bucket_size=bucket)
    w = np.random.default_rng(17).normal(0, 0.5 / p.n, p.n)
    check_eval(p, w, s)
    check_eval(p, w, s)   # second call runs from the neighbour cache


def test_eval_is_bit_reproducible_and_cache_independent(gpu):
    """Cached neighbour lists change the clipping order, not the result."""
    p = problems.make(1, g=48, res=192, beam=True)
    w1 = np.random.default_rng(5).normal(0, 0.5 / p.n, p.n)
    a = solver_for(p)
    f1, mu1, _, _ = a.eval(w1)          # cold: window candidates
    f2, mu2, _, _ = a.eval(w1)          # warm: cached neighbours
    b = solver_for(p)
    b.eval(np.zeros(p.n))               # cache from another point
    f3, mu3, _, _ = b.eval(w1)
    assert np.array_equal(mu1, mu2) and f1 == f2
    assert np.abs(mu1 - mu3).max() <= 1e-13 * mu1.max()


def test_large_instance_conservation(gpu):
    """Config-2 shape at full size: size-independent properties."""
    p = problems.make(2)
    s = solver_for(p)
    for w in (np.zeros(p.n), np.random.default_rng(2).normal(0, 0.5 / p.n, p.n)):
        f, mu, g, _ = s.eval(w)
        assert abs(mu.sum() - 1.0) < 1e-11
        assert abs(g.sum()) < 1e-11
        # adjacency is symmetric
        off, xy, nb = s.cells(w)
        pairs = set()
        for i in range(p.n):
            for j in nb[off[i]:off[i + 1]]:
                if j >= 0:
                    pairs.add((i, int(j)))
        assert all((j, i) in pairs for (i, j) in pairs)
    # directional derivative of f is g.d
    w = np.random.default_rng(3).normal(0, 0.5 / p.n, p.n)
    d = np.random.default_rng(4).normal(0, 1.0 / p.n, p.n)
    eps = 1e-3
    fp = s.eval(w + eps * d)[0]
    fm = s.eval(w - eps * d)[0]
    g = s.eval(w)[2]
    assert abs((fp - fm) / (2 * eps) - g @ d) < 1e-6 * abs(g @ d) + 1e-12


def test_wolfe_solve_matches_oracle(gpu):
    p = problems.make(1, g=16, res=64)
    s = solver_for(p)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    ow, ost = O.lbfgs_wolfe(oracle_problem(p), np.zeros(p.n), tol=1e-4, m=10)
    assert st.converged and ost.converged
    assert st.iterations == ost.iterations and st.evaluations == ost.evaluations
    # the two trajectories differ only by rounding (device reductions vs numpy
    # sums); over ~160 iterations that moves the weights far less than the
    # 1e-4 mass tolerance pins them (~1e-6 of their range)
    assert np.abs(w - ow).max() < 1e-6 * np.abs(ow).max()
    assert O.max_rel_error(O.evaluate(oracle_problem(p), w).mu, p.nu) <= 1e-4


def test_wolfe_solve_from_a_converged_start_stops_at_once(gpu):
    """The plain L-BFGS as the judge of a warm start: from weights that meet
    the tolerance it evaluates once and takes no iteration (the oracle's
    lbfgs_wolfe checks the start the same way), in both loops."""
    p = problems.make(1, g=16, res=64)
    s = solver_for(p)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-6, history=10)
    assert st.converged
    for use_graph in (0, -1):
        w2, st2 = s.solve(w, mode=capi.SOLVE_WOLFE, tol=1e-4, history=10, use_graph=use_graph)
        assert st2.converged and st2.iterations == 0 and st2.evaluations == 1
        assert np.array_equal(w2, w)
    _, ost = O.lbfgs_wolfe(oracle_problem(p), w, tol=1e-4, m=10)
    assert ost.converged and ost.iterations == 0 and ost.evaluations == 1


def test_wolfe_solve_passes_the_evaluation_noise_floor(gpu):
    """The device line search tolerates the objective's evaluation noise as
    the oracle does (approximate Wolfe): a small problem solves to 1e-10."""
    p = problems.make(2, 0, g=8, res=32)
    s = solver_for(p)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-10, history=10, max_iter=3000)
    assert st.converged and st.max_rel_err <= 1e-10
    assert O.max_rel_error(O.evaluate(oracle_problem(p), w).mu, p.nu) <= 1e-9


def test_reference_mode_solve_matches_oracle(gpu):
    """direct_ot's loop (backtracking, stale ||g|| stop) against its restatement."""
    p = problems.make(1, g=12, res=48)
    s = solver_for(p)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_REFERENCE, tol=1e-5, history=7, max_iter=2000)
    ow, ost = O.direct_ot_parity(oracle_problem(p), np.zeros(p.n), total_iter=2000, tol=1e-5, m=7)
    assert st.converged and ost.converged
    assert abs(st.iterations - ost.iterations) <= max(2, ost.iterations // 20)
    e = O.evaluate(oracle_problem(p), w)
    assert np.linalg.norm(e.g) < 2e-5


def test_reference_mode_first_divergence_is_a_rounding_tie(gpu):
    """Where the reference-mode trajectories of the device and the oracle
    part, the cause is a line-search decision on a tie: direct_ot accepts a
    trial when f(w + t d) < f_prev (ot_op.cuh:353-426), and at the first
    iteration whose accepted point differs, one of the two accepted points
    has an objective within the objective's evaluation noise of f_prev.  The
    two sides sum f in different orders (a fixed-order device reduction
    against the oracle's C loop), so such a comparison can go either way.
    Before that iteration the iterates agree to rounding."""
    p = problems.make(1, g=12, res=48)
    prob = oracle_problem(p)
    s = solver_for(p)
    gw = {}
    s.set_progress(lambda ph, it, stt, w, nu, gn, mr: gw.__setitem__(it, w), every=1)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_REFERENCE, tol=1e-5, history=7, max_iter=2000)
    ow = {}
    _, ost = O.direct_ot_parity(prob, np.zeros(p.n), total_iter=2000, tol=1e-5, m=7,
                                callback=lambda it, w_, fk, cur: ow.__setitem__(it, w_.copy()))
    its = sorted(set(gw) & set(ow))
    scale = max(np.abs(w).max(), 1e-300)
    first = next((k for k in its if np.abs(gw[k] - ow[k]).max() > 1e-6 * scale), None)
    if first is None:
        assert st.iterations == ost.iterations and st.evaluations == ost.evaluations
        return
    before = [k for k in its if k < first]
    assert before, "the trajectories part at the first iteration"
    prev = before[-1]
    assert np.abs(gw[prev] - ow[prev]).max() < 1e-9 * scale     # a jump, not a drift
    e_prev = O.evaluate(prob, ow[prev])
    noise = 1e-13 * np.abs(e_prev.fcell).sum()
    fg = O.evaluate(prob, gw[first]).f
    fo = O.evaluate(prob, ow[first]).f
    assert min(abs(fg - e_prev.f), abs(fo - e_prev.f)) <= noise, (first, fg - e_prev.f, fo - e_prev.f, noise)


def test_solve_reaches_tolerance_config1(gpu):
    p = problems.make(1)
    s = solver_for(p)
    w, st = s.solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    assert st.converged and st.max_rel_err <= 1e-4
    mu = O.evaluate(oracle_problem(p), w).mu
    assert O.max_rel_error(mu, p.nu) <= 1e-4 * (1 + 1e-6)
    assert abs(w.sum()) < 1e-12 * np.abs(w).sum()   # sum(g) = 0 keeps sum(w) (up to rounding)


def test_centroids_parity(gpu):
    p = problems.make(1, g=24, res=96)
    s = solver_for(p)
    w = np.random.default_rng(7).normal(0, 0.6 / p.n, p.n)
    c = O.cells(p.xy, w, O.proj_corner(p.xy, p.proj_domain))
    for weighted in (True, False):
        xy, ex = s.centroids(w, weighted=weighted)
        oxy, oex = O.centers(c, p.picture, p.size, p.proj_domain, weighting=weighted)
        assert np.array_equal(ex, oex)
        assert np.abs(xy[ex] - oxy[ex]).max() < 1e-10


def test_render_parity(gpu):
    """render (basic_function.cuh:660-741): nu spread over the pixels."""
    p = problems.make(1, g=20, res=80)
    s = solver_for(p)
    w = np.random.default_rng(9).normal(0, 0.5 / p.n, p.n)
    img = s.render(w, gray_multiple=1.0)
    c = O.cells(p.xy, w, O.proj_corner(p.xy, p.proj_domain))
    ref = O.render(c, p.nu, p.size, p.proj_domain)
    mu = s.eval(w)[1]
    assert abs(img.sum() - p.nu[mu > 0].sum()) < 1e-12   # hidden cells carry nothing
    assert np.abs(img - ref).max() < MU_TOL * ref.max()   # atomic accumulation order differs
    assert np.abs(s.render(w, gray_multiple=3.0) - 3.0 * img).max() < 1e-12 * img.max()


def test_source_masses_parity(gpu):
    pts = seeds.initial_xy_point(900, [0.0, 40.0, 0.0, 40.0])
    s = capi.Solver()
    nu = s.source_masses(pts, [0.0, 40.0, 0.0, 40.0])
    onu = O.source_masses(pts, [0.0, 40.0, 0.0, 40.0])
    assert abs(nu.sum() - 1600.0) < 1e-9
    assert np.abs(nu - onu).max() < 1e-10 * onu.max()


def test_point_light_source_masses_parity(gpu):
    """solid_angle (basic_function.cuh:558-588,635-658) source masses."""
    pts = seeds.initial_xy_point(400, [0.0, 40.0, 0.0, 40.0])
    light = [20.0, 20.0, -20.0]
    s = capi.Solver()
    nu = s.source_masses(pts, [0.0, 40.0, 0.0, 40.0], light=light, z_of_len=0.0)
    onu = O.source_masses_point_light(pts, [0.0, 40.0, 0.0, 40.0], light, 0.0)
    assert abs(nu.sum() - 1600.0) < 1e-9
    assert np.abs(nu - onu).max() < MU_TOL * onu.max()
    # cells right under the light see more of it than those in the corners
    c = np.argmin(np.hypot(pts[:, 0] - 20, pts[:, 1] - 20))
    assert nu[c] > nu[0]


def test_torch_device_buffers(gpu):
    import torch

    p = problems.make(1, g=16, res=64)
    s = capi.Solver()
    dev = torch.device("cuda", 0)
    s.set_problem(torch.from_numpy(p.xy.reshape(-1)).to(dev), torch.from_numpy(p.nu).to(dev),
                  torch.from_numpy(p.picture).to(dev), p.size, p.proj_domain)
    w = np.random.default_rng(1).normal(0, 0.3 / p.n, p.n)
    f, mu, g, fc = s.eval(torch.from_numpy(w).to(dev))
    ev = O.evaluate(oracle_problem(p), w)
    assert np.abs(mu.cpu().numpy() - ev.mu).max() <= MU_TOL * ev.mu.max()
    wd, st = s.solve(torch.zeros(p.n, dtype=torch.float64, device=dev), mode=capi.SOLVE_WOLFE, tol=1e-4)
    assert st.converged and wd.is_cuda


def test_set_up_from_host_and_device_arrays_agree(gpu):
    """cot_set_problem builds the problem on the device from host arrays
    (copied in first) or device arrays (read in place): the same bits."""
    import torch

    p = problems.make(1, g=40, res=160, beam=True)
    a = solver_for(p)
    b = capi.Solver()
    dev = torch.device("cuda", 0)
    b.set_problem(torch.from_numpy(p.xy.reshape(-1)).to(dev), torch.from_numpy(p.nu).to(dev),
                  torch.from_numpy(p.picture).to(dev), p.size, p.proj_domain)
    w = np.random.default_rng(31).normal(0, 0.5 / p.n, p.n)
    fa, mua, _, _ = a.eval(w)
    fb, mub, _, _ = b.eval(w)
    assert fa == fb and np.array_equal(mua, mub)
    wa, sa = a.solve(np.zeros(p.n), tol=1e-4)
    wb, sb = b.solve(np.zeros(p.n), tol=1e-4)
    assert np.array_equal(wa, wb) and sa.evaluations == sb.evaluations
    # a bad mass or pixel on the device is reported as on the host
    nu = torch.from_numpy(p.nu).to(dev)
    nu[17] = -1.0
    with pytest.raises(capi.CotError) as e:
        b.set_problem(torch.from_numpy(p.xy.reshape(-1)).to(dev), nu, torch.from_numpy(p.picture).to(dev), p.size,
                      p.proj_domain)
    assert "nu[17]" in str(e.value)
    pic = p.picture.copy()
    pic[99] = np.nan
    with pytest.raises(capi.CotError) as e:
        a.set_problem(p.xy, p.nu, pic, p.size, p.proj_domain)
    assert "pixel 99" in str(e.value)


def test_tiny_and_degenerate_inputs(gpu):
    """One site, two sites, sites on the domain boundary, a zero-density band."""
    dom = problems.UNIT_DOMAIN
    s = capi.Solver()
    s.set_problem(np.array([[0.3, 0.4]]), np.array([1.0]), np.ones(16), (4, 4), dom)
    f, mu, g, _ = s.eval(np.zeros(1))
    assert abs(mu[0] - 1.0) < 1e-14
    xy = np.array([[0.25, 0.5], [0.75, 0.5]])
    s.set_problem(xy, np.array([0.5, 0.5]), np.ones(16), (4, 4), dom)
    for dw in (0.0, 0.1, -0.05):
        mu = s.eval(np.array([dw, 0.0]))[1]
        assert abs(mu[0] - (0.5 + dw)) < 1e-14
    # sites on the boundary and a density with an empty band
    pts = np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0], [0.5, 0.5], [0.0, 0.5]])
    dens = np.ones((8, 8))
    dens[3:5, :] = 0.0
    nu = np.full(6, 1 / 6)
    s.set_problem(pts, nu, dens.ravel(), (8, 8), dom)
    w = np.array([0.0, 0.01, -0.01, 0.02, 0.0, 0.005])
    mu = s.eval(w)[1]
    prob = O.Problem(pts, nu, dens.ravel() / dens.sum(), (8, 8), dom)
    ev = O.evaluate(prob, w)
    assert np.abs(mu - ev.mu).max() < 1e-12


def test_bad_arguments_are_reported(gpu):
    s = capi.Solver()
    with pytest.raises(capi.CotError) as e:
        s.eval(np.zeros(4))
    assert e.value.code == capi.COT_ENOPROBLEM
    with pytest.raises(capi.CotError):
        s.set_problem(np.zeros((2, 2)), np.array([1.0, -1.0]), np.ones(4), (2, 2), problems.UNIT_DOMAIN)
    with pytest.raises(capi.CotError):
        s.set_problem(np.zeros((2, 2)), np.ones(2), np.ones(4), (2, 2), [1.0, 0.0, 0.0, 1.0])


def test_reference_run_on_gpu(gpu):
    """The committed reference run through the GPU path: source masses,
    masses at the converged weights and the weighted centroids."""
    with open(os.path.join(GOLD, "run.json")) as f:
        run = json.load(f)
    pts = seeds.initial_xy_point(run["point_num"], run["sample_domain"])
    proj = seeds.initial_proj_point(pts, run["sample_domain"], run["proj_domain"])
    pic = np.load(os.path.join(GOLD, "ustc_centerL.npz"))["picture"]
    dens, size = seeds.picture_from_matrix(pic)
    with gzip.open(os.path.join(GOLD, "weights0.txt.gz"), "rt") as f:
        w = np.loadtxt(f)
    s = capi.Solver()
    nu = s.source_masses(pts, run["sample_domain"])
    onu = O.source_masses(pts, run["sample_domain"])
    assert np.abs(nu - onu).max() < 1e-10 * onu.max()
    s.set_problem(proj, nu, dens, size, run["proj_domain"])
    f, mu, g, _ = s.eval(w)
    assert (mu == 0).sum() == 0
    assert np.linalg.norm(g) < 0.12
    pn = O.normalize_picture(dens, run["sample_domain"])
    ev = O.evaluate(O.Problem(proj, onu, pn, size, run["proj_domain"]), w)
    assert np.abs(mu - ev.mu).max() < 1e-10 * ev.mu.max()
    c, ex = s.centroids(w)
    assert ex.all()
    with gzip.open(os.path.join(GOLD, "out0_sub.txt.gz"), "rt") as f:
        sub = [r.split() for r in f.read().splitlines() if not r.startswith("#")]
    oi = np.array([int(a[0]) for a in sub])
    ov = np.array([[float(a[1]), float(a[2])] for a in sub])
    d = np.abs(c[oi] - ov)
    assert np.median(d) < 5e-4 and np.percentile(d, 99) < 1e-2 and d.max() < 3e-2


@pytest.mark.parametrize("mode", [capi.SOLVE_WOLFE, capi.SOLVE_REFERENCE])
def test_graph_loop_matches_host_loop(gpu, mode):
    """The device-driven trial loop (one CUDA graph, a WHILE node per trial)
    takes the same decisions as the host-driven one: same counts, same bits."""
    p = problems.make(1, g=24, res=96, beam=True)
    a = solver_for(p)
    wg, sg = a.solve(np.zeros(p.n), mode=mode, tol=1e-5 if mode == capi.SOLVE_REFERENCE else 1e-4, history=7,
                     max_iter=3000, use_graph=0)
    b = solver_for(p)
    wh, sh = b.solve(np.zeros(p.n), mode=mode, tol=1e-5 if mode == capi.SOLVE_REFERENCE else 1e-4, history=7,
                     max_iter=3000, use_graph=-1)
    assert sg.converged and sh.converged
    assert (sg.iterations, sg.evaluations, sg.restarts) == (sh.iterations, sh.evaluations, sh.restarts)
    assert np.array_equal(wg, wh)
    # the launch accounting of the graph counts every kernel of every pass
    ka, kb = a.kernel_stats(), b.kernel_stats()
    assert ka["evaluations"] == kb["evaluations"] and ka["cell_launches"] == kb["cell_launches"]
    # a solve cut short by max_iter stops at the same point
    wg2, sg2 = solver_for(p).solve(np.zeros(p.n), mode=mode, tol=1e-12, history=7, max_iter=37, use_graph=0)
    wh2, sh2 = solver_for(p).solve(np.zeros(p.n), mode=mode, tol=1e-12, history=7, max_iter=37, use_graph=-1)
    assert sg2.iterations == sh2.iterations == 37 and np.array_equal(wg2, wh2)


@pytest.mark.parametrize("cpw", [2, 4])
def test_two_cells_per_warp_parity(gpu, cpw):
    """16-lane (8-lane) segments, two (four) cells per warp: rings above 16
    (8) vertices go to a 32-lane pass and rings above 32 to the 256-vertex
    pass; a few heavy sites make giant cells so that every pass runs."""
    p = problems.make(1, g=32, res=128, beam=True)
    rng = np.random.default_rng(23)
    w = rng.normal(0, 0.3 / p.n, p.n)
    # five heavy sites spread over the domain: their cells spread over a few
    # pitches and keep most of the cells around them (rings of 16 to 40)
    order = np.argsort(p.xy[:, 0] * 7 + p.xy[:, 1])
    heavy = order[[150, 500, 850, 300, 700]]
    w[heavy[:3]] += 15.0 / p.n
    w[heavy[3:]] += 40.0 / p.n
    one = solver_for(p, cells_per_warp=1)
    two = solver_for(p, cells_per_warp=cpw)
    off, _, _ = two.cells(w)
    ring = np.diff(off)
    assert (ring > 16).sum() >= 3 and (ring > 32).sum() >= 2
    for _ in range(2):              # cold, then from the neighbour cache
        check_eval(p, w, two)
        f1, mu1, _, _ = one.eval(w)
        f2, mu2, _, _ = two.eval(w)
        assert np.abs(mu1 - mu2).max() <= 1e-13 * mu1.max()
    with pytest.raises(capi.CotError):
        capi.Solver(cells_per_warp=3)


@pytest.mark.parametrize("cpw", [2, 4])
def test_two_cells_per_warp_solve(gpu, cpw):
    p = problems.make(1, g=24, res=96, beam=True)
    w1, s1 = solver_for(p, cells_per_warp=1).solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    w2, s2 = solver_for(p, cells_per_warp=cpw).solve(np.zeros(p.n), mode=capi.SOLVE_WOLFE, tol=1e-4, history=10)
    assert s1.converged and s2.converged
    assert abs(s1.iterations - s2.iterations) <= max(3, s1.iterations // 20)
    # the 16-lane integration sums in another order: the trajectories part by
    # rounding, and both end inside the 1e-4 mass tolerance
    for w in (w1, w2):
        assert O.max_rel_error(O.evaluate(oracle_problem(p), w).mu, p.nu) <= 1e-4
    assert np.abs(w1 - w2).max() < 1e-4 * np.abs(w1).max()


def test_block_paths_match_oracle(gpu):
    """The paths that work one cell with several warps, against the oracle.
    Strongly weighted sites (cells far larger or smaller than their share,
    as early in a cold solve) give cells whose pixel box is large enough to
    have their integration started first or shared by several warps; with 2
    sites per bucket the bound tree is deep enough that certificate walks
    overflow their frontier, shrink their ring and, when they still
    overflow, are finished a block each.  Masses, gradient, objective and
    adjacency as in every evaluation test."""
    p = problems.make(1, g=64, res=1024)
    rng = np.random.default_rng(5)
    seen = {"walks_by_block": 0, "integrations_split": 0, "integrated_first": 0}
    for bucket_size in (16, 2):
        s = solver_for(p, bucket_size=bucket_size)
        for amp in (3.0, 10.0, 30.0):
            # the first evaluation at new weights: the cached rings of the
            # last weights mostly fail, as between far trial points
            w = rng.normal(0.0, amp / p.n, p.n)
            s.eval(w)
            c = s.eval_counters()
            for k in seen:
                seen[k] += c[k]
            check_eval(p, w, s)
        s.close()
    assert seen["walks_by_block"] > 0 and seen["integrations_split"] > 0 and seen["integrated_first"] > 0, seen
