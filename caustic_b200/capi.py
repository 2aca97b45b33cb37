"""ctypes binding of libcausticot.so (include/causticot.h).

The shared library is the product: every call here goes to the sm_100a CUDA
path.  There is no CPU fallback; if the library is missing or no GPU is
visible the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# CAUSTICOT_LIB selects another build of the same library (e.g. a measurement build)
LIB_PATH = os.environ.get("CAUSTICOT_LIB") or os.path.join(_PKG, "libcausticot.so")

COT_OK = 0
COT_EINVAL = -1
COT_ECUDA = -2
COT_ENOPROBLEM = -3
COT_ECAPACITY = -4
COT_ERING = -5
COT_ENOTCONV = -6
COT_ETIMEOUT = -7
COT_ENOMEM = -8
COT_ECANCELLED = -9

PHASE_LBFGS = 0
PHASE_PREPASS = 1
PHASE_ANDERSON = 2

COT_MEM_HOST = 0
COT_MEM_DEVICE = 1

SOLVE_REFERENCE = 0
SOLVE_WOLFE = 1

EXPORTED = [
    "cot_version", "cot_create", "cot_destroy", "cot_set_stream", "cot_set_problem", "cot_eval",
    "cot_cells", "cot_solve", "cot_centroids", "cot_source_masses", "cot_render", "cot_get_kernel_stats",
    "cot_eval_summary_noalloc", "cot_solve_aarl", "cot_source_masses_point_light", "cot_last_error",
    "cot_set_progress", "cot_solve_batch", "cot_solve_newton", "cot_mass_jacobian", "cot_eval_counters",
]
# int (*)(void *user, int phase, int iteration, int status, const double *w, const double *nu, int n,
#         double grad_norm, double max_rel_err)
PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                               ctypes.c_double, ctypes.c_double)
NOALLOC_MAX_N = 2048 * 1024


class cot_config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("bucket_size", ctypes.c_int),
                ("cells_per_warp", ctypes.c_int), ("max_ring", ctypes.c_int), ("profile", ctypes.c_int)]


class cot_kernel_stats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_longlong), ("cell_launches", ctypes.c_longlong),
                ("cell_ms", ctypes.c_double), ("evaluations", ctypes.c_longlong)]


class cot_solve_opts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("history", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("tol", ctypes.c_double), ("initial_step", ctypes.c_double), ("c1", ctypes.c_double),
                ("c2", ctypes.c_double), ("max_ls", ctypes.c_int), ("use_graph", ctypes.c_int)]


class cot_solve_stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("evaluations", ctypes.c_int), ("restarts", ctypes.c_int),
                ("converged", ctypes.c_int), ("f", ctypes.c_double), ("max_rel_err", ctypes.c_double),
                ("grad_norm", ctypes.c_double), ("empty_cells", ctypes.c_int),
                ("ring_overflows", ctypes.c_int), ("ms", ctypes.c_double)]


class cot_newton_opts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("cg_rtol", ctypes.c_double),
                ("cg_max_iter", ctypes.c_int), ("lbfgs_chunk", ctypes.c_int), ("lbfgs_rounds", ctypes.c_int),
                ("history", ctypes.c_int), ("shrink_steps", ctypes.c_int)]


class cot_newton_stats(ctypes.Structure):
    _fields_ = [("newton_iterations", ctypes.c_int), ("lbfgs_iterations", ctypes.c_int),
                ("evaluations", ctypes.c_int), ("cg_iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("fallback", ctypes.c_int), ("max_rel_err", ctypes.c_double), ("grad_norm", ctypes.c_double),
                ("empty_cells", ctypes.c_int), ("ms", ctypes.c_double)]


@dataclass
class NewtonStats:
    newton_iterations: int
    lbfgs_iterations: int
    evaluations: int
    cg_iterations: int
    converged: bool
    fallback: bool
    max_rel_err: float
    grad_norm: float
    empty_cells: int
    ms: float


class cot_aarl_inputs(ctypes.Structure):
    _fields_ = [("points_xy", ctypes.c_void_p), ("input_light", ctypes.c_void_p), ("inside_light", ctypes.c_void_p),
                ("height", ctypes.c_void_p), ("z_of_len", ctypes.c_double), ("z_of_receiver", ctypes.c_double),
                ("refraction_index", ctypes.c_double), ("sample_domain", ctypes.c_double * 4),
                ("aa_history", ctypes.c_int), ("aa_fixed_para", ctypes.c_double), ("lbfgs_prepass", ctypes.c_int)]


class CotError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"causticot error {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Load the shared library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m caustic_b200.build` (or "
                               "__graft_entry__.build()) first; there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        up = ctypes.POINTER(ctypes.c_ubyte)
        L.cot_version.argtypes = [ip, ip, ip]
        L.cot_create.argtypes = [ctypes.POINTER(cot_config), ctypes.POINTER(vp)]
        L.cot_destroy.argtypes = [vp]
        L.cot_set_stream.argtypes = [vp, vp]
        L.cot_set_problem.argtypes = [vp, vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        L.cot_eval.argtypes = [vp, vp, dp, vp, vp, vp, ctypes.c_int]
        L.cot_cells.argtypes = [vp, dp, ip, dp, ip, ctypes.c_int]
        L.cot_solve.argtypes = [vp, vp, ctypes.POINTER(cot_solve_opts), ctypes.POINTER(cot_solve_stats), ctypes.c_int]
        L.cot_centroids.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]
        L.cot_source_masses.argtypes = [vp, dp, ctypes.c_int, dp, dp]
        L.cot_source_masses_point_light.argtypes = [vp, dp, ctypes.c_int, dp, dp, ctypes.c_double, dp]
        L.cot_render.argtypes = [vp, dp, ctypes.c_double, dp]
        L.cot_get_kernel_stats.argtypes = [vp, ctypes.POINTER(cot_kernel_stats), ctypes.c_int]
        L.cot_eval_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.cot_eval_summary_noalloc.argtypes = [vp, vp, vp, ctypes.c_int, vp, vp]
        L.cot_solve_aarl.argtypes = [vp, vp, ctypes.POINTER(cot_aarl_inputs), ctypes.POINTER(cot_solve_opts),
                                     ctypes.POINTER(cot_solve_stats)]
        L.cot_solve_newton.argtypes = [vp, vp, ctypes.POINTER(cot_newton_opts), ctypes.POINTER(cot_newton_stats),
                                       ctypes.c_int]
        L.cot_mass_jacobian.argtypes = [vp, vp, ctypes.c_int, ip, ip, dp, ctypes.c_int, ip]
        L.cot_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
        L.cot_set_progress.argtypes = [vp, PROGRESS_FN, vp, ctypes.c_int]
        L.cot_solve_batch.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp),
                                      ctypes.POINTER(cot_solve_opts), ctypes.POINTER(cot_solve_stats)]
        for name in EXPORTED:
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _vptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def version():
    L = load()
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.cot_version(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


@dataclass
class SolveStats:
    iterations: int
    evaluations: int
    restarts: int
    converged: bool
    f: float
    max_rel_err: float
    grad_norm: float
    empty_cells: int
    ring_overflows: int
    ms: float


class Solver:
    """One handle: a problem on one GPU and the calls on it.

    Arrays may be numpy (host) or torch CUDA tensors (device, float64,
    contiguous); outputs come back in the same kind as the input weights.
    """

    def __init__(self, device: int = 0, bucket_size: int = 0, cells_per_warp: int = 0, max_ring: int = 0,
                 profile: bool = False):
        L = load()
        self._L = L
        cfg = cot_config(device, bucket_size, cells_per_warp, max_ring, int(bool(profile)))
        h = ctypes.c_void_p()
        rc = L.cot_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != COT_OK:
            raise CotError(rc, self._err(None))
        self._h = h
        self.n = 0
        self.device = device
        self._progress = None       # keeps the ctypes callback alive
        self._progress_exc = None   # exception raised inside the callback

    def set_progress(self, fn=None, every: int = 1):
        """Call fn(phase, iteration, status, w, nu, grad_norm, max_rel_err)
        after every iteration whose 0-based index is a multiple of `every`
        and after the last one of each phase (status 0 running, 1 converged,
        2 stopped; w, nu: numpy copies in caller order).  A truthy return
        stops the solve, which then returns its last iterate with
        converged=False.  fn may call eval / cells / centroids / render on
        this solver.  fn=None removes the callback."""
        if fn is None:
            self._check(self._L.cot_set_progress(self._h, PROGRESS_FN(), None, 1))
            self._progress = None
            return

        def tramp(user, phase, iteration, status, w, nu, n, gnorm, maxrel):
            try:
                wa = np.ctypeslib.as_array(w, shape=(n,)).copy()
                na = np.ctypeslib.as_array(nu, shape=(n,)).copy()
                return 1 if fn(phase, iteration, status, wa, na, gnorm, maxrel) else 0
            except BaseException as e:  # stop the solve, re-raise after it returns
                self._progress_exc = e
                return 1

        cb = PROGRESS_FN(tramp)
        self._check(self._L.cot_set_progress(self._h, cb, None, int(every)))
        self._progress = cb

    def _raise_progress_exc(self):
        e, self._progress_exc = self._progress_exc, None
        if e is not None:
            raise e

    def _err(self, h="self"):
        buf = ctypes.create_string_buffer(1024)
        self._L.cot_last_error(self._h if h == "self" else None, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc, allow=()):
        if rc != COT_OK and rc not in allow:
            raise CotError(rc, self._err())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            self._L.cot_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def kernel_stats(self, reset: bool = False) -> dict:
        """Launch counts and summed cell-kernel device time (profile=True)."""
        st = cot_kernel_stats()
        self._check(self._L.cot_get_kernel_stats(self._h, ctypes.byref(st), int(bool(reset))))
        return {"launches": st.launches, "cell_launches": st.cell_launches, "cell_ms": st.cell_ms,
                "evaluations": st.evaluations}

    def eval_counters(self) -> dict:
        """Slow paths taken by the last evaluation (cot_eval_counters)."""
        c = (ctypes.c_int * 4)()
        self._check(self._L.cot_eval_counters(self._h, c))
        return {"large_rings": c[0], "walks_by_block": c[1], "integrated_first": c[2],
                "integrations_split": c[3]}

    def set_stream(self, stream_ptr: int):
        self._check(self._L.cot_set_stream(self._h, ctypes.c_void_p(stream_ptr)))
        self._stream_ptr = int(stream_ptr or 0)

    def _order_after_torch(self, t):
        """Device tensors handed to the library were written on torch's
        current stream; unless the handle runs on that same stream, wait for
        it so that the library's stream reads them complete."""
        import torch

        cur = torch.cuda.current_stream(t.device)
        if getattr(self, "_stream_ptr", 0) == 0 or cur.cuda_stream != self._stream_ptr:
            cur.synchronize()

    # -------------------------------------------------------------------
    def set_problem(self, xy, nu, density, size, proj_domain):
        """size = (nx, ny): pixels along x and y, density[ix + iy*nx]."""
        nx, ny = int(size[0]), int(size[1])
        self._size = (nx, ny)
        pd = _f64(proj_domain)
        if _is_torch(xy):
            self._order_after_torch(xy)
            self._check(self._L.cot_set_problem(self._h, _tptr(xy), _tptr(nu), int(nu.numel()), _tptr(density),
                                                nx, ny, _dptr(pd), COT_MEM_DEVICE))
            self.n = int(nu.numel())
        else:
            xy, nu, density = _f64(xy), _f64(nu), _f64(density)
            self._keep = (xy, nu, density)
            self._check(self._L.cot_set_problem(self._h, _vptr(xy), _vptr(nu), int(nu.size), _vptr(density),
                                                nx, ny, _dptr(pd), COT_MEM_HOST))
            self.n = int(nu.size)

    def eval(self, w):
        """(f, mu, g, f_cell) at weights w."""
        f = ctypes.c_double()
        if _is_torch(w):
            import torch

            self._order_after_torch(w)
            mu = torch.empty_like(w)
            g = torch.empty_like(w)
            fc = torch.empty_like(w)
            rc = self._L.cot_eval(self._h, _tptr(w), ctypes.byref(f), _tptr(mu), _tptr(g), _tptr(fc),
                                  COT_MEM_DEVICE)
        else:
            w = _f64(w)
            mu, g, fc = np.empty_like(w), np.empty_like(w), np.empty_like(w)
            rc = self._L.cot_eval(self._h, _vptr(w), ctypes.byref(f), _vptr(mu), _vptr(g), _vptr(fc), COT_MEM_HOST)
        self._check(rc)
        return f.value, mu, g, fc

    def cells(self, w):
        """Rings of the cells inside proj_domain: (offsets[n+1], xy[V,2], nbr[V])."""
        w = _f64(w)
        cap = max(16 * self.n, 64)
        while True:
            off = np.zeros(self.n + 1, dtype=np.int32)
            xy = np.zeros(2 * cap)
            nb = np.zeros(cap, dtype=np.int32)
            rc = self._L.cot_cells(self._h, _dptr(w), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(xy),
                                   nb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cap)
            if rc == COT_ECAPACITY:
                cap *= 2
                continue
            self._check(rc)
            V = int(off[-1])
            return off, xy[: 2 * V].reshape(V, 2), nb[:V]

    def solve(self, w0, mode=SOLVE_WOLFE, history=10, max_iter=20000, tol=1e-4, initial_step=1.0,
              c1=0.0, c2=0.0, max_ls=0, use_graph=0, raise_on_noconv=False):
        opts = cot_solve_opts(mode, history, max_iter, tol, initial_step, c1, c2, max_ls, use_graph)
        st = cot_solve_stats()
        if _is_torch(w0):
            w = w0.clone()
            self._order_after_torch(w)
            rc = self._L.cot_solve(self._h, _tptr(w), ctypes.byref(opts), ctypes.byref(st), COT_MEM_DEVICE)
        else:
            w = _f64(w0).copy()
            rc = self._L.cot_solve(self._h, _vptr(w), ctypes.byref(opts), ctypes.byref(st), COT_MEM_HOST)
        self._raise_progress_exc()
        self._check(rc, allow=() if raise_on_noconv else (COT_ENOTCONV, COT_ECANCELLED))
        stats = SolveStats(st.iterations, st.evaluations, st.restarts, bool(st.converged), st.f, st.max_rel_err,
                           st.grad_norm, st.empty_cells, st.ring_overflows, st.ms)
        return w, stats

    def solve_newton(self, w0, tol=1e-4, max_iter=100, cg_rtol=0.1, cg_max_iter=2000, lbfgs_chunk=10,
                     lbfgs_rounds=50, history=10, shrink_steps=0, raise_on_noconv=False):
        """Damped Newton solve (cot_solve_newton): optionally a scaled-down
        start when the start empties cells (shrink_steps), L-BFGS while a cell
        is empty, then Newton steps on the masses' Jacobian; L-BFGS finishes
        if they stall.  Returns (weights, NewtonStats)."""
        opts = cot_newton_opts(tol, max_iter, cg_rtol, cg_max_iter, lbfgs_chunk, lbfgs_rounds, history,
                               shrink_steps)
        st = cot_newton_stats()
        if _is_torch(w0):
            w = w0.clone()
            self._order_after_torch(w)
            rc = self._L.cot_solve_newton(self._h, _tptr(w), ctypes.byref(opts), ctypes.byref(st), COT_MEM_DEVICE)
        else:
            w = _f64(w0).copy()
            rc = self._L.cot_solve_newton(self._h, _vptr(w), ctypes.byref(opts), ctypes.byref(st), COT_MEM_HOST)
        self._check(rc, allow=() if raise_on_noconv else (COT_ENOTCONV,))
        return w, NewtonStats(st.newton_iterations, st.lbfgs_iterations, st.evaluations, st.cg_iterations,
                              bool(st.converged), bool(st.fallback), st.max_rel_err, st.grad_norm, st.empty_cells,
                              st.ms)

    def mass_jacobian(self, w):
        """dmu/dw at w as a scipy CSR matrix (cot_mass_jacobian)."""
        import scipy.sparse as sp

        w = _f64(w)
        n = self.n
        off = np.zeros(n + 1, dtype=np.int32)
        nnz = ctypes.c_int(0)
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(self._L.cot_mass_jacobian(self._h, _vptr(w), COT_MEM_HOST, off.ctypes.data_as(ip), None, None,
                                              0, ctypes.byref(nnz)))
        cols = np.zeros(max(nnz.value, 1), dtype=np.int32)
        vals = np.zeros(max(nnz.value, 1))
        self._check(self._L.cot_mass_jacobian(self._h, _vptr(w), COT_MEM_HOST, off.ctypes.data_as(ip),
                                              cols.ctypes.data_as(ip), _dptr(vals), cols.size, ctypes.byref(nnz)))
        return sp.csr_matrix((vals[:nnz.value], cols[:nnz.value], off), shape=(n, n))

    def solve_aarl(self, w0, points, input_light, inside_light, height, *, z_of_len, z_of_receiver,
                   refraction_index, sample_domain, aa_history=7, aa_fixed_para=-2.0, lbfgs_prepass=True,
                   history=7, max_iter=50001, tol=0.01, initial_step=1.0, raise_on_noconv=False):
        """aarl_direct_ot: Fresnel-reweighted masses + Anderson acceleration.
        The problem's masses must be the source masses; on return they are
        the re-weighted ones.  Host arrays only."""
        w = _f64(w0).copy()
        keep = [_f64(points).reshape(-1), _f64(input_light).reshape(-1), _f64(inside_light).reshape(-1),
                _f64(height).reshape(-1)]
        ai = cot_aarl_inputs(keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data, keep[3].ctypes.data,
                             z_of_len, z_of_receiver, refraction_index,
                             (ctypes.c_double * 4)(*[float(v) for v in sample_domain]), aa_history, aa_fixed_para,
                             int(bool(lbfgs_prepass)))
        opts = cot_solve_opts(SOLVE_REFERENCE, history, max_iter, tol, initial_step, 0.0, 0.0, 0, 0)
        st = cot_solve_stats()
        rc = self._L.cot_solve_aarl(self._h, _vptr(w), ctypes.byref(ai), ctypes.byref(opts), ctypes.byref(st))
        self._raise_progress_exc()
        self._check(rc, allow=() if raise_on_noconv else (COT_ENOTCONV, COT_ECANCELLED))
        return w, SolveStats(st.iterations, st.evaluations, st.restarts, bool(st.converged), st.f, st.max_rel_err,
                             st.grad_norm, st.empty_cells, st.ring_overflows, st.ms)

    def centroids(self, w, weighted=True):
        if _is_torch(w):
            import torch

            self._order_after_torch(w)
            xy = torch.empty((self.n, 2), dtype=torch.float64, device=w.device)
            ex = torch.empty(self.n, dtype=torch.uint8, device=w.device)
            rc = self._L.cot_centroids(self._h, _tptr(w), _tptr(xy), _tptr(ex), int(bool(weighted)), COT_MEM_DEVICE)
            self._check(rc)
            return xy, ex.bool()
        w = _f64(w)
        xy = np.empty((self.n, 2))
        ex = np.empty(self.n, dtype=np.uint8)
        rc = self._L.cot_centroids(self._h, _vptr(w), _vptr(xy), _vptr(ex), int(bool(weighted)), COT_MEM_HOST)
        self._check(rc)
        return xy, ex.astype(bool)

    def render(self, w, gray_multiple=1.0, size=None):
        """render (basic_function.cuh:660-741): nu spread over the pixels,
        times gray_multiple; returns density-layout array nx*ny."""
        w = _f64(w)
        out = np.zeros(int(self._size[0]) * int(self._size[1]))
        self._check(self._L.cot_render(self._h, _dptr(w), float(gray_multiple), _dptr(out)))
        return out

    def source_masses(self, points, sample_domain, light=None, z_of_len=0.0):
        """Parallel light (light=None): cell areas; a point light: the solid
        angles of the cells seen from `light`; both normalised to the sample
        domain's area."""
        p = _f64(points).reshape(-1, 2)
        out = np.empty(p.shape[0])
        if light is None:
            rc = self._L.cot_source_masses(self._h, _dptr(p), p.shape[0], _dptr(_f64(sample_domain)), _dptr(out))
        else:
            rc = self._L.cot_source_masses_point_light(self._h, _dptr(p), p.shape[0], _dptr(_f64(sample_domain)),
                                                       _dptr(_f64(light)), float(z_of_len), _dptr(out))
        self._check(rc)
        return out


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _tptr(t):
    import torch

    if not t.is_cuda or t.dtype not in (torch.float64, torch.uint8) or not t.is_contiguous():
        raise ValueError("device arrays must be contiguous CUDA tensors (float64)")
    return ctypes.c_void_p(t.data_ptr())


def solve_batch(solvers, w0s, mode=SOLVE_WOLFE, history=10, max_iter=20000, tol=1e-4, initial_step=1.0, c1=0.0,
                c2=0.0, max_ls=0, raise_on_noconv=False):
    """Solve one problem per solver (all on one device) in a single graph
    launch on the first solver's stream (cot_solve_batch).  w0s: host start
    weights, one array per solver.  Returns (weights, stats), one entry per
    solver; every stats' ms is the time of the whole batch."""
    L = load()
    n = len(solvers)
    if n == 0 or len(w0s) != n:
        raise ValueError("one start vector per solver")
    ws = [_f64(w).copy() for w in w0s]
    for s_, w in zip(solvers, ws):
        if w.size != s_.n:
            raise ValueError("start vector of the wrong size")
    hs = (ctypes.c_void_p * n)(*[s_._h.value for s_ in solvers])
    wp = (ctypes.c_void_p * n)(*[w.ctypes.data for w in ws])
    opts = cot_solve_opts(mode, history, max_iter, tol, initial_step, c1, c2, max_ls, 0)
    st = (cot_solve_stats * n)()
    rc = L.cot_solve_batch(hs, n, wp, ctypes.byref(opts), st)
    solvers[0]._check(rc, allow=() if raise_on_noconv else (COT_ENOTCONV,))
    stats = [SolveStats(x.iterations, x.evaluations, x.restarts, bool(x.converged), x.f, x.max_rel_err, x.grad_norm,
                        x.empty_cells, x.ring_overflows, x.ms) for x in st]
    return ws, stats
