"""The warm-start network's kernels against the CPU restatement: the
tensor-core GEMMs, then forward, loss and every parameter gradient of a
small network; then that training lowers the loss and that the trained
network's starting point saves L-BFGS iterations."""
import numpy as np
import pytest

from caustic_b200 import problems, warmstart
from oracle import ws_oracle as R

pytestmark = pytest.mark.gpu


def bf16_tensor(torch, a):
    return torch.from_numpy(np.asarray(a, np.float32)).cuda().to(torch.bfloat16)


@pytest.mark.parametrize("layout", [warmstart.GEMM_RC, warmstart.GEMM_CR, warmstart.GEMM_RR])
def test_gemm_layouts(gpu, layout):
    import torch

    rng = np.random.default_rng(layout)
    M, N, K = 264, 40, 72          # not multiples of the 128x128x64 tile
    A = R.bf16(rng.normal(size=(M, K)))
    B = R.bf16(rng.normal(size=(K, N)))
    if layout == warmstart.GEMM_RC:
        a, b = A, B.T.copy()           # A [M][K], B stored [N][K]
    elif layout == warmstart.GEMM_CR:
        a, b = A.T.copy(), B           # A stored [K][M], B [K][N]
    else:
        a, b = A, B
    net = warmstart.WarmStartNet(levels=2, base=8)
    net._stream = torch.cuda.current_stream().cuda_stream
    D = torch.full((M, N), 0.5, dtype=torch.float32, device="cuda")
    net._gemm(layout, M, N, K, bf16_tensor(torch, a), bf16_tensor(torch, b), D, beta=1.0)
    ref = A @ B + 0.5
    assert np.abs(D.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()


def test_network_matches_oracle(gpu):
    import torch

    rng = np.random.default_rng(3)
    net = warmstart.WarmStartNet(levels=3, base=8, seed=4)
    for c in net.layers():          # non-zero biases so every path carries signal
        if c.b is not None:
            c.b.copy_(torch.from_numpy(rng.normal(0, 0.1, c.cout).astype(np.float32)))
    x = R.bf16(rng.normal(size=(2, 16, 16, warmstart.IN_CH)))
    t = rng.normal(size=(2, 256))
    pred = net.forward(bf16_tensor(torch, x), keep=True)
    loss, g = net.loss_grad(pred, torch.from_numpy(t.astype(np.float32)).cuda(), lam=5.0)
    net.zero_grad()
    net.backward(g)
    ref = R.Net([(c.w.cpu().numpy().astype(np.float64),
                  None if c.b is None else c.b.cpu().numpy().astype(np.float64)) for c in net.layers()],
                net.levels, net.ch)
    rp = ref.forward(x)
    rl, rg = R.loss_grad(rp, t, lam=5.0)
    grads = ref.backward(rg)
    p = pred.cpu().numpy()
    assert np.abs(p - rp).max() <= 2e-2 * np.abs(rp).max()
    assert abs(loss - rl) <= 2e-2 * rl
    for k, c in enumerate(net.layers()):
        gw, gb = grads[k]
        e = np.linalg.norm(c.gw.cpu().numpy() - gw) / max(np.linalg.norm(gw), 1e-30)
        assert e < 3e-2, (k, e)
        if gb is not None:
            eb = np.linalg.norm(c.gb.cpu().numpy() - gb) / max(np.linalg.norm(gb), 1e-30)
            assert eb < 3e-2, (k, eb)


def test_training_and_warm_start_gain(gpu):
    """Small instances (24x24 sites, 48^2 images): 256 solver-made pairs, a
    short training, then warm against cold solves of 16 held-out problems."""
    probs = [problems.make(4, i, g=24, res=48) for i in range(272)]
    train, held = probs[:256], probs[256:]
    ws, st = warmstart.solve_pairs(train, tol=1e-5)
    assert all(s.converged for s in st)
    net = warmstart.WarmStartNet(levels=3, base=16, seed=1)
    X = warmstart.make_input(train)
    Y, net.out_scale = warmstart.make_target(ws)
    hist = warmstart.fit(net, X, Y, epochs=80, batch=16, lr=2e-3)
    assert hist[-1] < 0.3 * hist[0]
    res = warmstart.compare(net, held, tol=1e-4)
    assert all(e <= 1e-4 for e in res["cold_err"] + res["warm_err"])
    # the network gets the large-scale transport right; the cells' masses
    # depend on the weights' differences at the pitch scale, which L-BFGS
    # still has to settle, so the saving is a fraction of the iterations
    assert np.mean(res["warm_iters"]) < 0.9 * np.mean(res["cold_iters"])
