"""ORACLE -- test infrastructure only.

CPU restatement of the reference semi-discrete OT solver of rmk523/caustic
(``Optimal_Transport_rl/``).  It is imported only by ``tests/``, by
``__graft_entry__.smoke()`` and by the CPU-baseline leg of ``bench.py``, and
there only as the checker.  The product (``caustic_b200`` over
``libcausticot.so``) never imports it.

Pieces:

* power-diagram topology: the regular triangulation of the weighted sites,
  taken from the lower convex hull of the lifted points (x, y, x^2+y^2-w)
  (Qhull through scipy).  This is the same triangulation the reference builds
  with CGAL 5.5 ``Regular_triangulation_2`` (power_diagram.cpp:51-52); CGAL is
  not present here, so its algorithm is restated rather than called.
* cell rings, per-cell integrals, centroids and source areas: the C library
  ``libsdot_oracle.so`` (``sdot_oracle.c``), which restates clip.cuh and
  basic_function.cuh in the reference operation order.
* the solver loops: ``direct_ot_parity`` restates ``direct_ot``
  (ot_op.cuh:66-589) step by step; ``lbfgs_wolfe`` is the configuration used by
  the benchmark configs (L-BFGS, strong-Wolfe line search, max-relative stop),
  written with the same update rules as the device solver.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsdot_oracle.so")
_lib = None
_lock = threading.Lock()

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_ubyte)


def build() -> str:
    """Compile the oracle C library with its committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE, "CC=gcc"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH) or (
                os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "sdot_oracle.c"))
            ):
                build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_eval_cells.argtypes = [ctypes.c_int, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp]
            L.orc_clip_area.argtypes = [ctypes.c_int, _dp, _ip, _ip, _dp, _dp]
            L.orc_edge_weights.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip, _ip, _dp, _dp, _ip, _dp, _dp]
            L.orc_center.argtypes = [ctypes.c_int, _dp, _ip, _ip, _dp, _ip, _dp, ctypes.c_int, _dp, _up]
            L.orc_render.argtypes = [ctypes.c_int, _dp, _ip, _ip, _dp, _ip, _dp, _dp]
            L.orc_cells.argtypes = [ctypes.c_int, _dp, _dp, _ip, _ip, _dp, ctypes.c_int, _ip, _dp, _ip]
            L.orc_cells_brute.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, _dp, _ip]
            L.orc_clip_rect.argtypes = [_dp, ctypes.c_int, _dp, _dp, _ip]
            L.orc_area.argtypes = [_dp, ctypes.c_int]
            L.orc_area.restype = ctypes.c_double
            L.orc_poly_ints.argtypes = [_dp, ctypes.c_int, _dp]
            L.orc_poly_ints.restype = ctypes.c_double
            _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# --------------------------------------------------------------------------
# topology
# --------------------------------------------------------------------------
def power_neighbors(xy: np.ndarray, w: np.ndarray):
    """Regular-triangulation neighbours of each site (CSR: start[n+1], nbr).

    Lower hull of the lifted points; sites that are not on it are hidden
    (empty power cell) and get no neighbours.
    """
    from scipy.spatial import ConvexHull

    xy = _f64(xy).reshape(-1, 2)
    n = xy.shape[0]
    if n < 4:
        # every pair is a candidate; the half-plane clip sorts it out
        nb = [np.array([j for j in range(n) if j != i], dtype=np.int32) for i in range(n)]
        start = np.zeros(n + 1, dtype=np.int32)
        start[1:] = np.cumsum([len(a) for a in nb])
        return start, (np.concatenate(nb) if n > 1 else np.zeros(0, np.int32))
    lifted = np.empty((n, 3))
    lifted[:, :2] = xy
    lifted[:, 2] = (xy * xy).sum(1) - _f64(w)
    hull = ConvexHull(lifted)
    low = hull.simplices[hull.equations[:, 2] < 0]
    e = np.concatenate([low[:, [0, 1]], low[:, [1, 2]], low[:, [2, 0]]])
    e = np.concatenate([e, e[:, ::-1]])
    e = np.unique(e, axis=0)
    start = np.zeros(n + 1, dtype=np.int64)
    np.add.at(start, e[:, 0] + 1, 1)
    start = np.cumsum(start).astype(np.int32)
    return start, _i32(e[:, 1])


def hidden_sites(start) -> np.ndarray:
    """Sites with no regular-triangulation neighbour: not on the lower hull,
    so their power cell is empty (CGAL leaves them out of the diagram and the
    reference writes length 0 for them, power_diagram.cpp:59-61)."""
    return np.diff(start) == 0


@dataclass
class Cells:
    """Fixed-stride rings: ring_xy[i, :ring_len[i]] (CCW), ring_lab the
    generator of edge k -> k+1 (site index, or -1..-4 for the box sides)."""

    ring_len: np.ndarray
    ring_xy: np.ndarray
    ring_lab: np.ndarray
    cap: int

    @property
    def start(self):
        return (np.arange(self.ring_len.shape[0], dtype=np.int32) * self.cap).astype(np.int32)

    def lens(self):
        return np.maximum(self.ring_len, 0).astype(np.int32)


def cells(xy, w, box, cap: int = 256, brute: bool = False) -> Cells:
    """Power cells intersected with box = {xmin, xmax, ymin, ymax}.

    restates polygons_in_VD (power_diagram.cpp:8-134) for the part of each
    ring inside the box; ring_len < 0 flags a ring above ``cap`` vertices.
    """
    L = lib()
    xy = _f64(xy).reshape(-1)
    w = _f64(w)
    n = w.shape[0]
    box = _f64(box)
    rl = np.zeros(n, dtype=np.int32)
    rx = np.zeros(2 * cap * max(n, 1), dtype=np.float64)
    rb = np.zeros(cap * max(n, 1), dtype=np.int32)
    if brute:
        L.orc_cells_brute(n, _d(xy), _d(w), _d(box), cap, _i(rl), _d(rx), _i(rb))
    else:
        st, nb = power_neighbors(xy.reshape(-1, 2), w)
        nb = _i32(nb) if nb.size else np.zeros(1, np.int32)
        L.orc_cells(n, _d(xy), _d(w), _i(_i32(st)), _i(nb), _d(box), cap, _i(rl), _d(rx), _i(rb))
        if n >= 4:
            rl[hidden_sites(st)] = 0
    return Cells(rl, rx.reshape(max(n, 1), cap, 2)[:n], rb.reshape(max(n, 1), cap)[:n], cap)


def adjacency(c: Cells, min_len: float = 0.0):
    """Set of (i, j), i < j, whose shared edge inside the box is longer than
    min_len; box sides excluded."""
    out = set()
    for i in range(c.ring_len.shape[0]):
        m = int(c.ring_len[i])
        if m <= 0:
            continue
        P = c.ring_xy[i, :m]
        Q = np.roll(P, -1, axis=0)
        ln = np.hypot(*(Q - P).T)
        for k in range(m):
            j = int(c.ring_lab[i, k])
            if j >= 0 and ln[k] > min_len:
                out.add((min(i, j), max(i, j)))
    return out


# --------------------------------------------------------------------------
# per-cell integrals
# --------------------------------------------------------------------------
def eval_cells(c: Cells, xy, w, nu, picture, size, proj_domain):
    """(mu, f_cell): compute_inte + compute_f (basic_function.cuh:743-952)."""
    L = lib()
    n = c.ring_len.shape[0]
    mu = np.zeros(n)
    f = np.zeros(n)
    rx = _f64(c.ring_xy).reshape(-1)
    L.orc_eval_cells(n, _d(rx), _i(c.start), _i(c.lens()), _d(_f64(xy).reshape(-1)), _d(_f64(w)),
                     _d(_f64(nu)), _d(_f64(picture).reshape(-1)), _i(_i32(size)), _d(_f64(proj_domain)),
                     _d(mu), _d(f))
    return mu, f


def edge_weights(c: Cells, xy, picture, size, proj_domain):
    """a[i, k] = (integral of the density along ring edge k of cell i) /
    (2 |s_i - s_j|) for an edge whose generator is a site j, else 0: the
    off-diagonal entries -dmu_i/dw_j of the masses' Jacobian (no counterpart
    in the reference; see orc_edge_weights)."""
    L = lib()
    n = c.ring_len.shape[0]
    out = np.zeros((n, c.cap))
    L.orc_edge_weights(n, c.cap, _d(_f64(c.ring_xy).reshape(-1)), _i(c.lens()), _i(_i32(c.ring_lab).reshape(-1)),
                       _d(_f64(xy).reshape(-1)), _d(_f64(picture).reshape(-1)), _i(_i32(size)),
                       _d(_f64(proj_domain)), _d(out.reshape(-1)))
    return out


def mass_jacobian(prob, w, c: Cells = None):
    """Sparse dmu/dw at w (scipy CSR, n x n): a weighted graph Laplacian,
    off-diagonal -a_ij from edge_weights, diagonal sum_j a_ij."""
    import scipy.sparse as sp

    if c is None:
        c = cells(prob.xy, w, prob.box, prob.cap)
    a = edge_weights(c, prob.xy, prob.picture, prob.size, prob.pd)
    n = prob.n
    lab = np.asarray(c.ring_lab)
    rows = np.repeat(np.arange(n), c.cap).reshape(n, c.cap)
    keep = (lab >= 0) & (a != 0.0)
    r, j, v = rows[keep], lab[keep].astype(np.int64), a[keep]
    H = sp.csr_matrix((-v, (r, j)), shape=(n, n))
    H = H + sp.diags(a.sum(axis=1))
    return H.tocsr()


def clip_area(c: Cells, sample_domain):
    L = lib()
    n = c.ring_len.shape[0]
    out = np.zeros(n)
    rx = _f64(c.ring_xy).reshape(-1)
    L.orc_clip_area(n, _d(rx), _i(c.start), _i(c.lens()), _d(_f64(sample_domain)), _d(out))
    return out


def centers(c: Cells, picture, size, proj_domain, weighting=True):
    L = lib()
    n = c.ring_len.shape[0]
    ctr = np.zeros(2 * n)
    ex = np.zeros(n, dtype=np.uint8)
    rx = _f64(c.ring_xy).reshape(-1)
    L.orc_center(n, _d(rx), _i(c.start), _i(c.lens()), _d(_f64(picture).reshape(-1)), _i(_i32(size)),
                 _d(_f64(proj_domain)), int(bool(weighting)), _d(ctr), ex.ctypes.data_as(_up))
    return ctr.reshape(n, 2), ex.astype(bool)


def render(c: Cells, carry, size, proj_domain):
    L = lib()
    n = c.ring_len.shape[0]
    out = np.zeros(int(size[0]) * int(size[1]))
    rx = _f64(c.ring_xy).reshape(-1)
    L.orc_render(n, _d(rx), _i(c.start), _i(c.lens()), _d(_f64(carry)), _i(_i32(size)),
                 _d(_f64(proj_domain)), _d(out))
    return out


# --------------------------------------------------------------------------
# problem set-up (ot_op.cuh:74-92, 154-206; main.cu:149-187)
# --------------------------------------------------------------------------
def normalize_picture(picture, sample_domain):
    """ot_op.cuh:81-88,154: picture /= (sum / area_scalar)."""
    sd = _f64(sample_domain)
    area_scalar = (sd[1] - sd[0]) * (sd[3] - sd[2])
    p = _f64(picture).reshape(-1)
    return p / (p.sum() / area_scalar)


def proj_corner(proj_xy, proj_domain):
    """main.cu:149-187."""
    xy = _f64(proj_xy).reshape(-1, 2)
    pd = _f64(proj_domain)
    xmn, xmx = xy[:, 0].min(), xy[:, 0].max()
    ymn, ymx = xy[:, 1].min(), xy[:, 1].max()
    c = [min(xmn, pd[0]), max(xmx, pd[1]), min(ymn, pd[2]), max(ymx, pd[3])]
    if c[0] == xmn:
        c[0] -= 1
    if c[1] == xmx:
        c[1] += 1
    if c[2] == ymn:
        c[2] -= 1
    if c[3] == ymx:
        c[3] += 1
    return np.array(c)


def source_masses(points, sample_domain):
    """Parallel-light source masses nu (ot_op.cuh:90-92,158,199-206).

    Unweighted power cells of the source points in the data_corner box
    (sample_domain pushed out by 1/40 of its extent), clipped to the sample
    domain, normalised to total area_scalar.
    """
    sd = _f64(sample_domain)
    xs, ys = sd[1] - sd[0], sd[3] - sd[2]
    corner = np.array([sd[0] - xs / 40, sd[1] + xs / 40, sd[2] - ys / 40, sd[3] + ys / 40])
    n = _f64(points).reshape(-1, 2).shape[0]
    c = cells(points, np.zeros(n), corner)
    a = clip_area(c, sd)
    return a / a.sum() * (xs * ys)


def solid_angle(poly, z, light):
    """compute_solid_angle (basic_function.cuh:558-588) of one ring."""
    L = _f64(light)
    P = np.column_stack([_f64(poly).reshape(-1, 2), np.full(len(poly), float(z))]) - L
    n = len(P)
    ang = 0.0
    for k in range(n - 2):
        v1 = P[0] / np.linalg.norm(P[0])
        v2 = P[k + 1] / np.linalg.norm(P[k + 1])
        v3 = P[k + 2] / np.linalg.norm(P[k + 2])
        num = float(v1 @ np.cross(v2, v3))
        den = 1.0 + float(v1 @ v2) + float(v2 @ v3) + float(v1 @ v3)
        if abs(den) < 1e-6:
            continue
        ang += 2 * np.arctan(num / den)
    return abs(ang)


def source_masses_point_light(points, sample_domain, light, z_of_len):
    """Point-light source masses (ot_op.cuh:160-206): solid angle of each
    source cell clipped to the sample domain, normalised to area_scalar."""
    L = lib()
    sd = _f64(sample_domain)
    xs, ys = sd[1] - sd[0], sd[3] - sd[2]
    corner = np.array([sd[0] - xs / 40, sd[1] + xs / 40, sd[2] - ys / 40, sd[3] + ys / 40])
    n = _f64(points).reshape(-1, 2).shape[0]
    c = cells(points, np.zeros(n), corner)
    sq = np.array([sd[0], sd[2], sd[1], sd[3]])
    out = np.zeros(2 * ORC_MAXD_PY)
    nn = ctypes.c_int()
    om = np.zeros(n)
    for i in range(n):
        m = int(c.ring_len[i])
        if m <= 0:
            continue
        ring = _f64(c.ring_xy[i, :m]).reshape(-1)
        L.orc_clip_rect(_d(ring), m, _d(sq), _d(out), ctypes.byref(nn))
        om[i] = solid_angle(out[: 2 * nn.value].reshape(-1, 2), z_of_len, light)
    return om / om.sum() * (xs * ys)


ORC_MAXD_PY = 512


# --------------------------------------------------------------------------
# evaluation bundle
# --------------------------------------------------------------------------
@dataclass
class Problem:
    """Sites, target masses and density in the reference's conventions.

    picture: already normalised (sum = area of the sample domain), layout
    picture[ix + iy*size[0]]; pd = proj_domain {xmin, xmax, ymin, ymax};
    box = the box the raw rings are bounded by (proj_corner)."""

    xy: np.ndarray
    nu: np.ndarray
    picture: np.ndarray
    size: np.ndarray
    pd: np.ndarray
    box: np.ndarray = None
    cap: int = 256

    def __post_init__(self):
        self.xy = _f64(self.xy).reshape(-1, 2)
        self.nu = _f64(self.nu)
        self.picture = _f64(self.picture).reshape(-1)
        self.size = _i32(self.size)
        self.pd = _f64(self.pd)
        if self.box is None:
            self.box = proj_corner(self.xy, self.pd)
        self.box = _f64(self.box)

    @property
    def n(self):
        return self.xy.shape[0]


@dataclass
class Eval:
    f: float
    mu: np.ndarray
    g: np.ndarray
    fcell: np.ndarray
    max_len: int
    cells: Cells = None


def evaluate(prob: Problem, w, keep_cells=False) -> Eval:
    c = cells(prob.xy, w, prob.box, prob.cap)
    max_len = int(c.ring_len.max()) if c.ring_len.size else 0
    if (c.ring_len < 0).any():
        max_len = prob.cap + 1
    mu, fc = eval_cells(c, prob.xy, w, prob.nu, prob.picture, prob.size, prob.pd)
    return Eval(float(fc.sum()), mu, mu - prob.nu, fc, max_len, c if keep_cells else None)


# --------------------------------------------------------------------------
# solvers
# --------------------------------------------------------------------------
@dataclass
class SolveStats:
    iterations: int = 0
    evaluations: int = 0
    restarts: int = 0
    converged: bool = False
    history: list = field(default_factory=list)


def direct_ot_parity(prob: Problem, w0, total_iter=50001, tol=0.01, initial_step=1.0, m=7,
                     max_ring=200, callback=None):
    """Restatement of direct_ot's L-BFGS loop (ot_op.cuh:289-537).

    Backtracking with simple decrease, the polygon-complexity reject
    (ring > max_edge_num/2 = 200), the restart at step <= 1e-4*initial_step,
    and the stop on the stale ||g||_2 with no empty cell.
    """
    w = _f64(w0).copy()
    n = w.shape[0]
    st = SolveStats()
    ev = evaluate(prob, w)
    st.evaluations += 1
    fk, mu, g = ev.f, ev.mu, ev.g
    S = np.zeros((m, n))
    Y = np.zeros((m, n))
    rho = np.zeros(m)
    alpha = np.zeros(m)
    H0 = 1.0
    restart = False
    loop_iter = 0
    for it in range(total_iter):
        max_idx = min(loop_iter, m)
        d = -g
        poly_inte = mu.copy()
        deri = g.copy()
        if not restart:
            for i in range(1, max_idx + 1):
                idx = (loop_iter - i) % m
                alpha[idx] = float((S[idx] * d).sum()) * rho[idx]
                d = d + (-alpha[idx]) * Y[idx]
            d = d * H0
            for i in range(max_idx, 0, -1):
                idx = (loop_iter - i) % m
                beta = rho[idx] * float((Y[idx] * d).sum())
                d = d + (alpha[idx] - beta) * S[idx]
        if float((g * d).sum()) >= 0:
            d = -g
            loop_iter = 0
            H0 = 1.0
        gkm1 = g.copy()
        wm1 = w.copy()
        fkm1 = fk
        step = initial_step
        while True:
            w = wm1 + step * d
            ev = evaluate(prob, w)
            st.evaluations += 1
            if ev.max_len > max_ring:
                step *= 0.5
            else:
                fk = ev.f
                if fk < fkm1:
                    mu, g = ev.mu, ev.g
                    restart = False
                    break
                step *= 0.5
            if step <= 1e-4 * initial_step:
                restart = True
                g = gkm1
                loop_iter = 0
                H0 = 1.0
                w = wm1
                fk = fkm1
                st.restarts += 1
                break
        st.iterations = it + 1
        if step <= 1e-4 * initial_step:
            continue
        h = loop_iter % m
        S[h] = step * d
        Y[h] = g - gkm1
        ys = float((Y[h] * S[h]).sum())
        yy = float((Y[h] * Y[h]).sum())
        with np.errstate(divide='ignore', invalid='ignore'):
            rho[h] = np.float64(1.0) / np.float64(ys)   # C++ semantics: 1/0 -> inf
        H0 = ys / yy if yy > 1e-5 else 1.0
        loop_iter += 1
        cur = float(np.linalg.norm(deri))
        degen = int((poly_inte == 0).sum())
        st.history.append((fk, cur, degen, step))
        if callback:
            callback(it, w, fk, cur)
        if cur < tol and degen == 0:
            st.converged = True
            break
    return w, st


def max_rel_error(mu, nu):
    return float(np.max(np.abs(mu - nu) / nu))


F_NOISE = 1e-12  # relative objective noise the Wolfe search tolerates (COT_F_NOISE)


def lbfgs_wolfe(prob: Problem, w0, tol=1e-4, m=10, max_iter=20000, c1=1e-4, c2=0.9,
                max_ls=30, max_ring=None, max_evals=None):
    """L-BFGS with a strong-Wolfe line search and the max-relative mass stop.

    Same rules as the device solver (caustic_b200 csrc/cot_solver.cu):
    first trial step 1 (unit step on the scaled direction), bracketing by
    doubling, zoom by bisection; a change of f within F_NOISE |f| is not
    held against a step whose slope is small enough (approximate Wolfe); the
    history pair is stored only when y.s > 0; the stop test
    max_i |mu_i - nu_i| / nu_i <= tol is taken at the accepted point.
    """
    w = _f64(w0).copy()
    n = w.shape[0]
    st = SolveStats()
    ev = evaluate(prob, w)
    st.evaluations += 1
    f, mu, g = ev.f, ev.mu, ev.g
    S = np.zeros((m, n))
    Y = np.zeros((m, n))
    rho = np.zeros(m)
    k = 0
    H0 = 1.0
    for it in range(max_iter):
        err = max_rel_error(mu, prob.nu)
        st.history.append((f, err))
        if err <= tol:
            st.converged = True
            break
        if max_evals is not None and st.evaluations >= max_evals:
            break
        q = -g
        cnt = min(k, m)
        alpha = np.zeros(m)
        for i in range(1, cnt + 1):
            idx = (k - i) % m
            alpha[idx] = rho[idx] * float(S[idx] @ q)
            q = q - alpha[idx] * Y[idx]
        q = q * H0
        for i in range(cnt, 0, -1):
            idx = (k - i) % m
            beta = rho[idx] * float(Y[idx] @ q)
            q = q + (alpha[idx] - beta) * S[idx]
        d = q
        gd = float(g @ d)
        if gd >= 0:
            d = -g
            gd = float(g @ d)
            k = 0
            H0 = 1.0
        # strong Wolfe: bracket by doubling, then bisect
        lo, hi = 0.0, np.inf
        f_lo, t = f, 1.0
        e_lo = None
        acc = None
        for _ in range(max_ls):
            if max_evals is not None and st.evaluations >= max_evals:
                break
            wt = w + t * d
            e = evaluate(prob, wt)
            st.evaluations += 1
            bad = max_ring is not None and e.max_len > max_ring
            gtd = float(e.g @ d)
            # approximate Wolfe (cot_solver.cu ls_decide): a change of f
            # within F_NOISE |f| (evaluation noise) does not count against
            # the step when the slope g(t).d <= (2 c1 - 1) g.d
            approx = e.f <= f + F_NOISE * abs(f) and gtd <= (2.0 * c1 - 1.0) * gd
            if bad or (not approx and (e.f > f + c1 * t * gd or e.f >= f_lo)):
                hi = t
            elif abs(gtd) <= c2 * abs(gd):
                acc = (t, e)
                break
            elif gtd > 0:
                hi = t
            else:
                # an approximate-Wolfe step may sit a rounding above f_lo:
                # it moves lo but never raises f_lo (as cot_solver.cu)
                lo, f_lo, e_lo = t, min(f_lo, e.f), e
            t = 2.0 * t if not np.isfinite(hi) else 0.5 * (lo + hi)
        if acc is None:
            if lo > 0:
                acc = (lo, e_lo)
            else:
                st.restarts += 1
                k = 0
                H0 = 1.0
                if st.restarts > 50:
                    break
                continue
        t, e = acc
        s = t * d
        y = e.g - g
        ys = float(y @ s)
        w = w + s
        f, mu, g = e.f, e.mu, e.g
        if ys > 0:
            h = k % m
            S[h], Y[h], rho[h] = s, y, 1.0 / ys
            H0 = ys / float(y @ y)
            k += 1
        st.iterations = it + 1
    return w, st


# --------------------------------------------------------------------------
# aarl_direct_ot (ot_op.cuh:591-1385)
# --------------------------------------------------------------------------
def _normalize3(v):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        out = np.where(n < 1e-12, 0.0, v / n)
    return out


def _fresnel_t(wi, wt, nrm, eta_i, eta_t):
    """fresnel_T_unpolarized, basic_function.cuh:407-435 (rows of vectors)."""
    eps = 1e-12
    ci = np.clip(np.abs((wi * nrm).sum(-1)), 0.0, 1.0)
    ct = np.clip(np.abs((wt * nrm).sum(-1)), 0.0, 1.0)
    ds = eta_i * ci + eta_t * ct
    dp = eta_i * ct + eta_t * ci
    ds = np.where(np.abs(ds) < eps, eps, ds)
    dp = np.where(np.abs(dp) < eps, eps, dp)
    rs = ((eta_i * ci - eta_t * ct) / ds) ** 2
    rp = ((eta_i * ct - eta_t * ci) / dp) ** 2
    return 1.0 - 0.5 * (rs + rp)


def energy_remain_rate(points, z_len, input_light, inside_light, height, out_points, z_recv, eta):
    """compute_energy_remain_rate, basic_function.cuh:437-494."""
    pts = _f64(points).reshape(-1, 2)
    n = pts.shape[0]
    p = np.column_stack([pts, np.full(n, z_len)])
    wi = _f64(input_light).reshape(-1, 3)
    ins = _f64(inside_light).reshape(-1, 3)
    op = p + _f64(height)[:, None] * ins
    rec = np.column_stack([_f64(out_points).reshape(-1, 2), np.full(n, z_recv)])
    wt = _normalize3(rec - op)
    n2 = _normalize3(eta * ins - wt)
    n1 = np.tile([0.0, 0.0, 1.0], (n, 1))
    return _fresnel_t(wi, ins, n1, 1.0, eta) * _fresnel_t(ins, wt, n2, eta, 1.0)


def aarl_direct_ot(prob: Problem, w0, lam, points, input_light, inside_light, height, z_len, z_recv, eta,
                   aa_history=7, aa_fixed_para=-2.0, prepass=True, total_iter=50001, tol=0.01, m=7,
                   initial_step=1.0, max_ring=200):
    """Restatement of aarl_direct_ot.  lam: source masses (sum = area_scalar).
    Cells that do not exist take their site as the centroid (the reference
    reads whatever the centroid buffer held there)."""
    lam = _f64(lam)
    total = lam.sum()
    st = SolveStats()

    def nu_at(w):
        c = cells(prob.xy, w, prob.box, prob.cap)
        ctr, ex = centers(c, prob.picture, prob.size, prob.pd, weighting=False)
        ctr = np.where(ex[:, None], ctr, prob.xy)
        e = lam * energy_remain_rate(points, z_len, input_light, inside_light, height, ctr, z_recv, eta)
        return e / e.sum() * total, c

    w = _f64(w0).copy()
    prob.nu, _ = nu_at(w)
    if prepass:
        w, pre = direct_ot_parity(prob, w, total_iter=total_iter, tol=tol, initial_step=initial_step, m=m,
                                  max_ring=max_ring)
        st.evaluations += pre.evaluations
        prob.nu, _ = nu_at(w)
    ev = evaluate(prob, w)
    mu, g = ev.mu, ev.g
    M = aa_history
    n = w.shape[0]
    Gh = np.zeros((M, n))
    Fh = np.zeros((M, n))
    aa = 0
    for it in range(total_iter):
        cnt = min(aa + 1, M)
        h = aa % M
        empty_start = int((mu == 0).sum())
        Gh[h] = g
        Fh[h] = w + aa_fixed_para * g
        A = Gh[:cnt] @ Gh[:cnt].T + 1e-10 * np.eye(cnt)
        a = np.linalg.solve(A, np.ones(cnt))
        a = a / a.sum()
        d = a @ Fh[:cnt] - w
        t = 1.0
        acc = False
        while True:
            wt = w + t * d
            c = cells(prob.xy, wt, prob.box, prob.cap)
            st.evaluations += 1
            if c.ring_len.max() > max_ring or (c.ring_len < 0).any():
                t *= 0.5
            else:
                prob.nu, _ = nu_at(wt)
                mu_t, _ = eval_cells(c, prob.xy, wt, prob.nu, prob.picture, prob.size, prob.pd)
                w, mu, g = wt, mu_t, mu_t - prob.nu
                aa += 1
                acc = True
                break
            if t <= 1e-4 * initial_step:
                break
        if not acc:
            aa = 0
            st.restarts += 1
        st.iterations = it + 1
        check = empty_start if it % 10 == 0 else 0
        if np.linalg.norm(g) < tol and check == 0:
            st.converged = True
            break
    return w, prob.nu.copy(), st
