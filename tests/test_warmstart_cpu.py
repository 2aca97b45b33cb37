"""The warm-start network without a GPU: its CPU restatement's gradients
against finite differences (the oracle the GPU gradients are checked
against), and the kernel library's exports against its header."""
import ctypes
import os
import re

import numpy as np

from caustic_b200 import build, warmstart
from oracle import ws_oracle as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_gradients_match_finite_differences(monkeypatch):
    monkeypatch.setattr(R, "bf16", lambda x: np.asarray(x, np.float64))   # exact arithmetic
    rng = np.random.default_rng(0)
    levels, ch = 2, [8, 16]
    shapes = [(8, 72), (8, 72), (16, 72), (16, 144), (8, 216), (8, 72), (8, 8)]
    params = [(rng.normal(0, 0.3, s), None if k == len(shapes) - 1 else rng.normal(0, 0.1, s[0]))
              for k, s in enumerate(shapes)]
    net = R.Net(params, levels, ch)
    x = rng.normal(size=(2, 4, 4, 8))
    t = rng.normal(size=(2, 16))
    loss, g = R.loss_grad(net.forward(x), t)
    grads = net.backward(g)
    for k in (0, 3, 4, 6):
        w, b = params[k]
        for idx in [(0, 0), (w.shape[0] - 1, w.shape[1] - 1), (min(3, w.shape[0] - 1), 5)]:
            old = w[idx]
            w[idx] = old + 1e-6
            lp, _ = R.loss_grad(net.forward(x), t)
            w[idx] = old - 1e-6
            lm, _ = R.loss_grad(net.forward(x), t)
            w[idx] = old
            fd = (lp - lm) / 2e-6
            assert abs(fd - grads[k][0][idx]) <= 1e-6 * max(1.0, abs(fd)), (k, idx)
        if b is not None:
            old = b[0]
            b[0] = old + 1e-6
            lp, _ = R.loss_grad(net.forward(x), t)
            b[0] = old - 1e-6
            lm, _ = R.loss_grad(net.forward(x), t)
            b[0] = old
            assert abs((lp - lm) / 2e-6 - grads[k][1][0]) <= 1e-6 * max(1.0, abs(grads[k][1][0]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], np.float64)
    r = R.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 1e-3) <= 2 ** -9 * 1e-3


def test_kernel_library_exports_its_header():
    build.build_ws()
    with open(os.path.join(ROOT, "include", "causticws.h")) as f:
        names = re.findall(r"WS_API\s+\w+\s+((?:ws|cot_warmstart)_\w+)\s*\(", f.read())
    assert "ws_gemm" in names and "ws_adam" in names
    lib = ctypes.CDLL(warmstart.WS_LIB)
    assert not [n for n in names if not hasattr(lib, n)]


def test_loss_with_neighbour_term_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.normal(size=(2, 12))
    t = rng.normal(size=(2, 12))
    loss, g = R.loss_grad(p, t, grid=(3, 4), lam=2.5)
    for idx in [(0, 0), (0, 5), (1, 11), (1, 6)]:
        q = p.copy()
        q[idx] += 1e-6
        lp, _ = R.loss_grad(q, t, grid=(3, 4), lam=2.5)
        q[idx] -= 2e-6
        lm, _ = R.loss_grad(q, t, grid=(3, 4), lam=2.5)
        assert abs((lp - lm) / 2e-6 - g[idx]) <= 1e-7
    # a constant shift of a prediction changes nothing
    l2, _ = R.loss_grad(p + np.array([[3.0], [-1.0]]), t, grid=(3, 4), lam=2.5)
    assert abs(l2 - loss) <= 1e-12
