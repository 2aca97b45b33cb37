"""Fresnel-reweighted Anderson solve (aarl_direct_ot, ot_op.cuh:591-1385):
GPU path against the oracle's restatement."""
import numpy as np
import pytest

from caustic_b200 import capi, problems
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def inputs(p, seed=5):
    rng = np.random.default_rng(seed)
    n = p.n
    pts = p.xy * 40.0
    inl = np.tile([0.0, 0.0, 1.0], (n, 1))
    insl = np.column_stack([rng.normal(0, 0.05, n), rng.normal(0, 0.05, n), np.ones(n)])
    insl /= np.linalg.norm(insl, axis=1, keepdims=True)
    hgt = rng.uniform(5, 10, n)
    return pts, inl, insl, hgt


def test_fresnel_rate_matches_reference_formula():
    """Straight-through light (no refraction at normal incidence) keeps
    (1 - R)^2 with R = ((n-1)/(n+1))^2 (basic_function.cuh:407-494)."""
    n = 4
    pts = np.zeros((n, 2))
    inl = np.tile([0.0, 0.0, 1.0], (n, 1))
    out = np.zeros((n, 2))
    t = O.energy_remain_rate(pts, 0.0, inl, inl, np.ones(n), out, 10.0, 1.5)
    R = ((1.5 - 1) / (1.5 + 1)) ** 2
    assert np.allclose(t, (1 - R) ** 2, rtol=1e-14)


def test_aarl_matches_oracle(gpu):
    p = problems.make(1, g=12, res=48)
    pts, inl, insl, hgt = inputs(p)
    kw = dict(aa_history=7, aa_fixed_para=-0.3, total_iter=300, tol=3e-6, m=7)
    prob = O.Problem(p.xy, p.nu.copy(), p.picture, p.size, p.proj_domain)
    ow, onu, ost = O.aarl_direct_ot(prob, np.zeros(p.n), p.nu, pts, inl, insl, hgt, 0.0, 3.0, 1.5, prepass=True, **kw)
    assert ost.converged
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = s.solve_aarl(np.zeros(p.n), pts, inl, insl, hgt, z_of_len=0.0, z_of_receiver=3.0, refraction_index=1.5,
                         sample_domain=[0, 40, 0, 40], aa_history=7, aa_fixed_para=-0.3, lbfgs_prepass=True,
                         history=7, max_iter=300, tol=3e-6)
    assert st.converged
    assert st.grad_norm < 3e-6
    assert abs(st.iterations - ost.iterations) <= max(5, ost.iterations // 4)
    # masses re-weighted at the GPU's weights: GPU vs oracle at the same point
    f, mu, g, _ = s.eval(w)
    nu_gpu = mu - g
    prob2 = O.Problem(p.xy, p.nu.copy(), p.picture, p.size, p.proj_domain)
    c = O.cells(p.xy, w, prob2.box)
    ctr, ex = O.centers(c, p.picture, p.size, p.proj_domain, weighting=False)
    ctr = np.where(ex[:, None], ctr, p.xy)
    e = p.nu * O.energy_remain_rate(pts, 0.0, inl, insl, hgt, ctr, 3.0, 1.5)
    nu_or = e / e.sum() * p.nu.sum()
    assert np.abs(nu_gpu - nu_or).max() < 1e-10 * nu_or.max()
    assert abs(nu_gpu.sum() - 1.0) < 1e-12


def test_aarl_without_prepass_runs(gpu):
    p = problems.make(1, g=10, res=40)
    pts, inl, insl, hgt = inputs(p, 7)
    s = capi.Solver()
    s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = s.solve_aarl(np.zeros(p.n), pts, inl, insl, hgt, z_of_len=0.0, z_of_receiver=3.0, refraction_index=1.5,
                         sample_domain=[0, 40, 0, 40], aa_history=5, aa_fixed_para=-0.3, lbfgs_prepass=False,
                         history=7, max_iter=40, tol=1e-12)
    assert not st.converged and st.iterations == 40
    assert np.isfinite(w).all() and st.grad_norm < 0.05
