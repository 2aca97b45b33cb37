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


def test_every_layer_matches_oracle_on_its_own_inputs(gpu):
    """Layer by layer, on the GPU's own inputs to each layer (so BF16
    rounding flips of earlier layers do not compound): forward
    pre-activations, each weight and bias gradient, and each input gradient
    agree with float64 sums of the same BF16 operands to 1e-5 (FP32
    accumulation is the only difference), and the bf16 operands of the
    backward GEMMs are bit-identical."""
    import torch

    rng = np.random.default_rng(8)
    net = warmstart.WarmStartNet(levels=3, base=8, seed=5)
    for c in net.layers():
        if c.b is not None:
            c.b.copy_(torch.from_numpy(rng.normal(0, 0.1, c.cout).astype(np.float32)))
    x = R.bf16(rng.normal(size=(2, 16, 16, warmstart.IN_CH)))
    t = rng.normal(size=(2, 256))
    net.trace = []
    pred = net.forward(bf16_tensor(torch, x), keep=True)
    tape = [(c, cols.double().cpu().numpy(), None if pre is None else pre.double().cpu().numpy())
            for (c, cols, pre, hh, ww) in net._tape[0]]
    loss, g = net.loss_grad(pred, torch.from_numpy(t.astype(np.float32)).cuda())
    net.zero_grad()
    net.backward(g)
    TOL = 1e-5

    def rel(a, b):
        return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)

    for c, cols, pre in tape:
        W = R.bf16(c.w.cpu().numpy().astype(np.float64))
        d = cols @ W.T
        if pre is not None:
            assert rel(pre, d + c.b.cpu().numpy()) < TOL
        else:
            assert rel(pred.double().cpu().numpy().reshape(-1), d[:, 0]) < TOL
    cols_of = {id(c): cols for c, cols, _ in tape}
    pre_of = {id(c): pre for c, _, pre in tape}
    assert len(net.trace) == len(tape)
    for c, dy, dz, dx in net.trace:
        dy = dy.double().cpu().numpy()
        dz = dz.double().cpu().numpy()
        pre = pre_of[id(c)]
        if pre is not None:
            # bias + ReLU backward, then the bf16 rounding of the GEMM operand
            assert np.array_equal(dz, R.bf16(dy * (pre > 0)))
            assert rel(c.gb.double().cpu().numpy(), (dy * (pre > 0)).sum(axis=0)) < TOL
        else:
            assert np.array_equal(dz, R.bf16(dy))
        assert rel(c.gw.double().cpu().numpy(), dz.T @ cols_of[id(c)]) < TOL
        dcols = dz @ R.bf16(c.w.cpu().numpy().astype(np.float64))
        if c.k == 3:
            M = dz.shape[0]
            side = int(round(np.sqrt(M // 2)))
            exp = R.col2im(dcols, (2, side, side, c.cin)).reshape(M, c.cin)
        else:
            exp = dcols
        assert rel(dx.double().cpu().numpy(), exp) < TOL


def test_c_abi_predict_matches_python(gpu, tmp_path):
    """cot_warmstart_predict (a C caller's learned start) gives the Python
    host layer's prediction: same inputs, same kernels, same weights."""
    import torch

    rng = np.random.default_rng(12)
    net = warmstart.WarmStartNet(levels=3, base=8, seed=9)
    for c in net.layers():
        if c.b is not None:
            c.b.copy_(torch.from_numpy(rng.normal(0, 0.1, c.cout).astype(np.float32)))
    net.out_scale = 3.7
    path = str(tmp_path / "net.bin")
    net.save_bin(path)
    cn = warmstart.CNet(path)
    for p in (problems.make(2, 3, g=16, res=64), problems.make(4, 5, g=32, res=64)):
        ref = warmstart.predict(net, [p])[0]
        got = cn.predict(p)
        assert np.abs(got - ref).max() <= 1e-3 * np.abs(ref).max()
    with pytest.raises(RuntimeError):
        cn.predict(problems.make(4, 5, g=10, res=40))   # 10 is not a multiple of 2^(levels-1) = 4
    cn.close()
