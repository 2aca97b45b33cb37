"""cot_eval_summary_noalloc: the allocation-free summary for callers that may
not call cudaMalloc (code recording a stream capture, hosts with a fixed
memory budget).  Its results must equal what the allocating path (cot_eval)
reports, on consecutive calls that reuse the shared scratch array.

Kept in a file of its own that is collected last.
"""
import ctypes

import numpy as np
import pytest

from caustic_b200 import capi, problems

pytestmark = pytest.mark.gpu

F_TOL = 1e-9       # objective: same tolerance as the parity tests
STAT_TOL = 1e-12   # statistics of identical per-cell arrays


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_summary_matches_cot_eval(gpu):
    import torch

    lib = capi.load()
    p = problems.make(1, g=40, res=160, beam=True)
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    dev = torch.device("cuda", 0)
    nu_d = torch.from_numpy(p.nu).to(dev)
    rng = np.random.default_rng(21)
    # two calls in a row, at two different points, through the same scratch
    for k in range(2):
        w = rng.normal(0.0, (0.3 + k) / p.n, p.n)
        f, mu, g, fc = s.eval(w)                      # the allocating entry point
        mu_d = torch.from_numpy(mu).to(dev)
        fc_d = torch.from_numpy(fc).to(dev)
        out = torch.full((4,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.cot_eval_summary_noalloc(_ptr(mu_d), _ptr(fc_d), _ptr(nu_d), p.n, _ptr(out), None)
        assert rc == capi.COT_OK
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        assert abs(o[0] - f) <= F_TOL * max(abs(f), np.abs(fc).sum())
        ref_rel = np.max(np.abs(g) / p.nu)
        assert abs(o[1] - ref_rel) <= STAT_TOL * ref_rel
        ref_g2 = float(g @ g)
        assert abs(o[2] - ref_g2) <= STAT_TOL * ref_g2 + 1e-300
        assert o[3] == float((mu == 0).sum())


def test_noalloc_rejects_oversize_and_null(gpu):
    import torch

    lib = capi.load()
    dev = torch.device("cuda", 0)
    a = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.cot_eval_summary_noalloc(_ptr(a), _ptr(a), _ptr(a), capi.NOALLOC_MAX_N + 1, _ptr(a), None)
    assert rc == capi.COT_EINVAL
    buf = ctypes.create_string_buffer(256)
    lib.cot_last_error(None, buf, 256)
    assert b"COT_NOALLOC_MAX_N" in buf.value
    assert lib.cot_eval_summary_noalloc(None, _ptr(a), _ptr(a), 8, _ptr(a), None) == capi.COT_EINVAL


def test_noalloc_nan_mass_is_not_converged(gpu):
    """A NaN among the masses must not vanish from the max-relative error
    (a plain fmax would drop it and the summary would look converged)."""
    import torch

    lib = capi.load()
    dev = torch.device("cuda", 0)
    n = 5000
    nu = torch.full((n,), 1.0 / n, dtype=torch.float64, device=dev)
    mu = nu.clone()
    mu[1234] = float("nan")
    fc = torch.zeros(n, dtype=torch.float64, device=dev)
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert lib.cot_eval_summary_noalloc(_ptr(mu), _ptr(fc), _ptr(nu), n, _ptr(out), None) == capi.COT_OK
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    assert o[1] == np.inf
