"""Learned warm start for the SDOT solve.

A convolutional encoder-decoder (U-Net, ``levels`` levels of two 3x3
convolutions with ReLU, channels ``base * 2**l``) maps a target image and the
site layout to initial dual weights on the site grid.  The plain L-BFGS
(``capi.Solver.solve``) then runs from them to the same tolerance: the
network only moves the starting point; the solver alone decides when the
error is small enough.

Every layer runs on the kernels of ``libcausticws.so`` (include/causticws.h):
im2col + a BF16 tensor-core GEMM with FP32 accumulation for the convolutions,
and hand-written kernels for bias + ReLU, pooling, upsampling, skip
connections, the loss and Adam.  torch only provides device buffers and the
input preparation.

Inputs (NHWC, 8 channels at the site grid's resolution, site grid G_x x G_y):
  0: log of the target density (pixels averaged onto the site grid),
     centred per image;
  1, 2: each site's jitter from its grid point, in quarter pitches;
  3: log(N * nu_i), each site's mass against the uniform 1/N (zero for
     uniform masses, so a network trained on those alone sees no change);
  4..7: zero (channel padding for the GEMM's 16-byte rows).
Output: N * w / out_scale (weights scaled by the number of sites and by the
spread of the training targets, stored with the network), compared with the
solver's weights after removing each one's mean.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
WS_LIB = os.environ.get("CAUSTICWS_LIB") or os.path.join(_PKG, "libcausticws.so")
IN_CH = 8
GEMM_RC, GEMM_CR, GEMM_RR = 0, 1, 2
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(WS_LIB):
            raise RuntimeError(f"{WS_LIB} is missing: run `python -m caustic_b200.build` first; there is no CPU "
                               "fallback")
        L = ctypes.CDLL(WS_LIB)
        vp, i, ll, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
        L.ws_gemm.argtypes = [i, i, i, i, vp, vp, vp, f, f, vp, ctypes.c_size_t, vp]
        L.ws_gemm_workspace.argtypes = [i, i, i, i]
        L.ws_gemm_workspace.restype = ctypes.c_size_t
        L.ws_im2col.argtypes = [i, i, i, i, vp, vp, vp]
        L.ws_col2im.argtypes = [i, i, i, i, vp, vp, vp]
        L.ws_bias_act.argtypes = [ll, i, vp, vp, i, vp, vp, vp]
        L.ws_act_back.argtypes = [ll, i, vp, vp, vp, vp, vp]
        L.ws_colsum.argtypes = [ll, i, vp, vp, vp]
        L.ws_pool2.argtypes = [i, i, i, i, vp, vp, vp]
        L.ws_pool2_back.argtypes = [i, i, i, i, vp, vp, vp]
        L.ws_up2.argtypes = [i, i, i, i, vp, i, i, vp, vp]
        L.ws_up2_back.argtypes = [i, i, i, i, vp, i, i, vp, vp]
        L.ws_put_channels.argtypes = [ll, i, vp, i, i, vp, vp]
        L.ws_take_channels.argtypes = [ll, i, vp, i, i, i, vp, vp]
        L.ws_mse_centered.argtypes = [i, i, i, f, vp, vp, vp, vp, vp]
        L.ws_adam.argtypes = [ll, vp, vp, vp, vp, vp, f, f, f, f, i, vp]
        L.ws_to_bf16.argtypes = [ll, vp, vp, vp]
        for name in ("ws_gemm", "ws_im2col", "ws_col2im", "ws_bias_act", "ws_act_back", "ws_colsum", "ws_pool2",
                     "ws_pool2_back", "ws_up2", "ws_up2_back", "ws_put_channels", "ws_take_channels",
                     "ws_mse_centered", "ws_adam", "ws_to_bf16"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc}")


@dataclass
class Conv:
    """3x3 convolution (or 1x1 when k == 1), weights [cout][k*k*cin]."""
    cin: int
    cout: int
    k: int = 3
    relu: bool = True
    w: object = None      # fp32 master
    w16: object = None    # bf16 copy for the GEMMs
    b: object = None      # fp32 bias (None for the head)
    gw: object = None
    gb: object = None
    state: list = field(default_factory=list)   # Adam moments


class WarmStartNet:
    """U-Net on the site grid; see the module docstring."""

    def __init__(self, levels: int = 4, base: int = 32, seed: int = 0, device: str = "cuda"):
        import torch

        self.torch = torch
        self.dev = torch.device(device)
        self.levels = levels
        self.ch = [base * (2 ** l) for l in range(levels)]
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.enc: List[List[Conv]] = []
        cin = IN_CH
        for l in range(levels):
            self.enc.append([Conv(cin, self.ch[l]), Conv(self.ch[l], self.ch[l])])
            cin = self.ch[l]
        self.dec: List[List[Conv]] = []
        for l in range(levels - 2, -1, -1):
            self.dec.append([Conv(self.ch[l + 1] + self.ch[l], self.ch[l]), Conv(self.ch[l], self.ch[l])])
        # 1x1 head to 8 outputs (16-byte rows), of which channel 0 is used;
        # no bias: the loss and the solve ignore a constant shift
        self.head = Conv(self.ch[0], 8, k=1, relu=False)
        for c in self.layers():
            fan = c.k * c.k * c.cin
            w = torch.randn(c.cout, fan, generator=g) * np.sqrt(2.0 / fan)
            if c is self.head:
                w[1:] = 0.0
            c.w = w.to(self.dev, torch.float32).contiguous()
            c.w16 = c.w.to(torch.bfloat16)
            c.b = None if c is self.head else torch.zeros(c.cout, device=self.dev, dtype=torch.float32)
            c.gw = torch.zeros_like(c.w)
            c.gb = None if c.b is None else torch.zeros_like(c.b)
            c.state = [torch.zeros_like(c.w), torch.zeros_like(c.w)] + (
                [] if c.b is None else [torch.zeros_like(c.b), torch.zeros_like(c.b)])
        self.step = 0
        self.out_scale = 1.0  # N * w = out_scale * output
        # set to a list to record, per backward layer, (conv, dy, dz, dx): the
        # incoming gradient, the bf16 gradient the GEMMs read and the result
        self.trace = None
        self._ws = None
        self._ws_bytes = 0

    def layers(self):
        for pair in self.enc:
            yield from pair
        for pair in self.dec:
            yield from pair
        yield self.head

    # -- parameters -------------------------------------------------------
    def state_dict(self) -> dict:
        out = {"levels": np.array(self.levels), "base": np.array(self.ch[0]), "out_scale": np.array(self.out_scale)}
        for k, c in enumerate(self.layers()):
            out[f"w{k}"] = c.w.cpu().numpy()
            if c.b is not None:
                out[f"b{k}"] = c.b.cpu().numpy()
        return out

    def load_state_dict(self, sd: dict):
        torch = self.torch
        self.out_scale = float(sd.get("out_scale", 1.0))
        for k, c in enumerate(self.layers()):
            c.w.copy_(torch.from_numpy(np.asarray(sd[f"w{k}"], np.float32)))
            c.w16.copy_(c.w.to(torch.bfloat16))
            if c.b is not None:
                c.b.copy_(torch.from_numpy(np.asarray(sd[f"b{k}"], np.float32)))

    def save_bin(self, path: str):
        """The flat binary that cot_warmstart_load (include/causticws.h) reads:
        "CWS1", int32 levels, base, layer count, float64 out_scale, then per
        layer (encoder, decoder, head) int32 cout, cin, k, has_bias and its
        float32 weights [cout][k*k*cin] and biases [cout]."""
        import struct

        layers = list(self.layers())
        with open(path, "wb") as f:
            f.write(b"CWS1")
            f.write(struct.pack("<iiid", self.levels, self.ch[0], len(layers), float(self.out_scale)))
            for c in layers:
                f.write(struct.pack("<iiii", c.cout, c.cin, c.k, 0 if c.b is None else 1))
                f.write(np.ascontiguousarray(c.w.cpu().numpy(), np.float32).tobytes())
                if c.b is not None:
                    f.write(np.ascontiguousarray(c.b.cpu().numpy(), np.float32).tobytes())

    @classmethod
    def from_file(cls, path: str, device: str = "cuda"):
        sd = dict(np.load(path))
        net = cls(levels=int(sd["levels"]), base=int(sd["base"]), device=device)
        net.load_state_dict(sd)
        return net

    # -- building blocks --------------------------------------------------
    def _workspace(self, need: int):
        if need > self._ws_bytes:
            self._ws = self.torch.empty(max(need, 1), dtype=self.torch.uint8, device=self.dev)
            self._ws_bytes = need
        return self._ws

    def _gemm(self, layout, M, N, K, A, B, D, beta=0.0):
        L = load()
        need = L.ws_gemm_workspace(layout, M, N, K)
        ws = self._workspace(need)
        _ok(L.ws_gemm(layout, M, N, K, _p(A), _p(B), _p(D), 1.0, beta, _p(ws) if need else None, need,
                      self._stream), f"gemm {layout} {M}x{N}x{K}")

    def _conv_fwd(self, c: Conv, x, Bn, H, W):
        torch = self.torch
        L = load()
        M = Bn * H * W
        if c.k == 3:
            cols = torch.empty(M, 9 * c.cin, dtype=torch.bfloat16, device=self.dev)
            _ok(L.ws_im2col(Bn, H, W, c.cin, _p(x), _p(cols), self._stream), "im2col")
        else:
            cols = x.view(M, c.cin)
        d = torch.empty(M, c.cout, dtype=torch.float32, device=self.dev)
        self._gemm(GEMM_RC, M, c.cout, c.k * c.k * c.cin, cols, c.w16, d)
        if c.b is None:
            return d, cols, None
        y = torch.empty(M, c.cout, dtype=torch.bfloat16, device=self.dev)
        pre = torch.empty(M, c.cout, dtype=torch.float32, device=self.dev)
        _ok(L.ws_bias_act(M, c.cout, _p(d), _p(c.b), 1 if c.relu else 0, _p(y), _p(pre), self._stream), "bias_act")
        return y, cols, pre

    def _conv_bwd(self, c: Conv, dy, cols, pre, Bn, H, W):
        """dy: fp32 [M, cout].  Accumulates c.gw, c.gb; returns dx fp32."""
        torch = self.torch
        L = load()
        M = Bn * H * W
        K = c.k * c.k * c.cin
        dz = torch.empty(M, c.cout, dtype=torch.bfloat16, device=self.dev)
        if pre is not None:
            dz32 = torch.empty(M, c.cout, dtype=torch.float32, device=self.dev)
            _ok(L.ws_act_back(M * c.cout, 1 if c.relu else 0, _p(dy), _p(pre), _p(dz), _p(dz32), self._stream),
                "act_back")
            gb = torch.empty_like(c.gb)
            _ok(L.ws_colsum(M, c.cout, _p(dz32), _p(gb), self._stream), "colsum")
            c.gb += gb
        else:
            _ok(L.ws_to_bf16(M * c.cout, _p(dy), _p(dz), self._stream), "to_bf16")
        self._gemm(GEMM_CR, c.cout, K, M, dz, cols, c.gw, beta=1.0)
        dcols = torch.empty(M, K, dtype=torch.float32, device=self.dev)
        self._gemm(GEMM_RR, M, K, c.cout, dz, c.w16, dcols)
        if c.k == 1:
            if self.trace is not None:
                self.trace.append((c, dy.clone(), dz.clone(), dcols.clone()))
            return dcols
        dx = torch.empty(M, c.cin, dtype=torch.float32, device=self.dev)
        _ok(L.ws_col2im(Bn, H, W, c.cin, _p(dcols), _p(dx), self._stream), "col2im")
        if self.trace is not None:
            self.trace.append((c, dy.clone(), dz.clone(), dx.clone()))
        return dx

    # -- network ----------------------------------------------------------
    def forward(self, x, keep: bool = False):
        """x: bf16 [B, H, W, 8] with H, W divisible by 2**(levels-1).
        Returns fp32 [B, H*W] (N * w up to a constant)."""
        torch = self.torch
        L = load()
        self._stream = torch.cuda.current_stream(self.dev).cuda_stream
        Bn, H, W, _ = x.shape
        tape = []
        skips = []
        h, hh, ww = x.contiguous(), H, W
        for l in range(self.levels):
            for c in self.enc[l]:
                y, cols, pre = self._conv_fwd(c, h, Bn, hh, ww)
                tape.append((c, cols, pre, hh, ww))
                h = y
            skips.append((h, hh, ww))
            if l < self.levels - 1:
                p = torch.empty(Bn, hh // 2, ww // 2, self.ch[l], dtype=torch.bfloat16, device=self.dev)
                _ok(L.ws_pool2(Bn, hh, ww, self.ch[l], _p(h), _p(p), self._stream), "pool2")
                h, hh, ww = p, hh // 2, ww // 2
        for j, l in enumerate(range(self.levels - 2, -1, -1)):
            ct = self.ch[l + 1] + self.ch[l]
            cat = torch.empty(Bn, hh * 2, ww * 2, ct, dtype=torch.bfloat16, device=self.dev)
            _ok(L.ws_up2(Bn, hh, ww, self.ch[l + 1], _p(h), ct, 0, _p(cat), self._stream), "up2")
            sk, sh, sw = skips[l]
            _ok(L.ws_put_channels(Bn * sh * sw, self.ch[l], _p(sk), ct, self.ch[l + 1], _p(cat), self._stream),
                "put_channels")
            h, hh, ww = cat, sh, sw
            for c in self.dec[j]:
                y, cols, pre = self._conv_fwd(c, h, Bn, hh, ww)
                tape.append((c, cols, pre, hh, ww))
                h = y
        d, cols, _ = self._conv_fwd(self.head, h, Bn, hh, ww)
        tape.append((self.head, cols, None, hh, ww))
        pred = d[:, 0].contiguous().view(Bn, hh * ww)
        if keep:
            self._tape = (tape, Bn, H, W)
        return pred

    def backward(self, dpred):
        """dpred: fp32 [B, H*W], gradient of the loss w.r.t. forward()'s
        output.  Accumulates the parameter gradients."""
        torch = self.torch
        L = load()
        tape, Bn, H, W = self._tape
        t = len(tape) - 1
        c, cols, pre, hh, ww = tape[t]
        dd = torch.zeros(Bn * hh * ww, 8, dtype=torch.float32, device=self.dev)
        dd[:, 0] = dpred.reshape(-1)
        dh = self._conv_bwd(c, dd, cols, pre, Bn, hh, ww)
        t -= 1
        dskip = [None] * self.levels
        # decoder, last level first
        dec_levels = list(range(self.levels - 2, -1, -1))
        for j in range(len(dec_levels) - 1, -1, -1):
            l = dec_levels[j]
            for _ in range(2):
                c, cols, pre, hh, ww = tape[t]
                dh = self._conv_bwd(c, dh, cols, pre, Bn, hh, ww)
                t -= 1
            ct = self.ch[l + 1] + self.ch[l]
            ds = torch.empty(Bn * hh * ww, self.ch[l], dtype=torch.float32, device=self.dev)
            _ok(L.ws_take_channels(Bn * hh * ww, self.ch[l], _p(dh), ct, self.ch[l + 1], 0, _p(ds), self._stream),
                "take_channels")
            dskip[l] = ds
            du = torch.empty(Bn * (hh // 2) * (ww // 2), self.ch[l + 1], dtype=torch.float32, device=self.dev)
            _ok(L.ws_up2_back(Bn, hh // 2, ww // 2, self.ch[l + 1], _p(dh), ct, 0, _p(du), self._stream), "up2_back")
            dh = du
        # encoder, deepest level first
        for l in range(self.levels - 1, -1, -1):
            hh = H >> l
            ww = W >> l
            if l < self.levels - 1:
                dp = torch.empty(Bn * hh * ww, self.ch[l], dtype=torch.float32, device=self.dev)
                _ok(L.ws_pool2_back(Bn, hh, ww, self.ch[l], _p(dh), _p(dp), self._stream), "pool2_back")
                dh = dp + dskip[l]
            for _ in range(2):
                c, cols, pre, ch_, cw_ = tape[t]
                dh = self._conv_bwd(c, dh, cols, pre, Bn, ch_, cw_)
                t -= 1
        assert t == -1
        self._tape = None
        return dh

    def zero_grad(self):
        for c in self.layers():
            c.gw.zero_()
            if c.gb is not None:
                c.gb.zero_()

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = load()
        self.step += 1
        for c in self.layers():
            if c is self.head:
                c.gw[1:] = 0.0
            _ok(L.ws_adam(c.w.numel(), _p(c.w), _p(c.w16), _p(c.gw), _p(c.state[0]), _p(c.state[1]), lr, b1, b2, eps,
                          self.step, self._stream), "adam")
            if c.b is not None:
                _ok(L.ws_adam(c.b.numel(), _p(c.b), None, _p(c.gb), _p(c.state[2]), _p(c.state[3]), lr, b1, b2, eps,
                              self.step, self._stream), "adam")

    def loss_grad(self, pred, target, grid=None, lam: float = 0.0):
        """Mean-free squared error on the site grid (ws_mse_centered), with
        lam weighing the neighbour differences: (loss, dpred).  grid =
        (gy, gx), default square."""
        torch = self.torch
        L = load()
        Bn, n = pred.shape
        gy, gx = grid if grid else (int(round(np.sqrt(n))),) * 2
        if gy * gx != n:
            raise ValueError("grid does not match the prediction")
        grad = torch.empty_like(pred)
        lb = torch.empty(Bn, dtype=torch.float32, device=self.dev)
        _ok(L.ws_mse_centered(Bn, gy, gx, float(lam), _p(pred), _p(target.contiguous()), _p(grad), _p(lb),
                              self._stream), "mse")
        return float(lb.sum()), grad


# ---------------------------------------------------------------------------
# inputs and targets
# ---------------------------------------------------------------------------
def make_input(probs, device="cuda"):
    """bf16 NHWC [B, G_y, G_x, 8] for problems on a G_x x G_y jittered grid
    whose image is a multiple of the grid (see the module docstring)."""
    import torch

    xs = []
    for p in probs:
        gx, gy = p.grid
        W, H = p.size
        fy, fx = H // gy, W // gx
        img = np.asarray(p.picture, np.float64).reshape(H, W)
        img = img.reshape(gy, fy, gx, fx).mean(axis=(1, 3)) * (H * W)
        lg = np.log(np.maximum(img, 1e-12))
        lg -= lg.mean()
        u = (np.arange(gx) + 0.5) / gx
        v = (np.arange(gy) + 0.5) / gy
        jx = (p.xy[:, 0].reshape(gy, gx) - u[None, :]) * (4 * gx)
        jy = (p.xy[:, 1].reshape(gy, gx) - v[:, None]) * (4 * gy)
        x = np.zeros((gy, gx, IN_CH), np.float32)
        x[..., 0] = lg
        x[..., 1] = jx
        x[..., 2] = jy
        x[..., 3] = np.log(np.maximum(np.asarray(p.nu, np.float64) * p.n, 1e-300)).reshape(gy, gx)
        xs.append(x)
    return torch.from_numpy(np.stack(xs)).to(device=device, dtype=torch.bfloat16)


def make_target(ws, scale: float = 0.0, device="cuda"):
    """(fp32 [B, N] device tensor, scale): N * w with its mean removed,
    divided by scale (0: the targets' own standard deviation)."""
    import torch

    t = np.stack([np.asarray(w, np.float64) * len(w) for w in ws])
    t -= t.mean(axis=1, keepdims=True)
    if not scale > 0:
        scale = float(t.std()) or 1.0
    return torch.from_numpy((t / scale).astype(np.float32)).to(device), scale


def predict(net: WarmStartNet, probs, batch: int = 32) -> list:
    """Initial weights (host float64, mean zero) for each problem."""
    out = []
    for k in range(0, len(probs), batch):
        part = probs[k:k + batch]
        pred = net.forward(make_input(part, net.dev)).double().cpu().numpy()
        for p, row in zip(part, pred):
            w = row * net.out_scale / p.n
            out.append(w - w.mean())
    return out


class CNet:
    """The network through the C ABI (cot_warmstart_load / _predict, the
    same entry points a C caller binds): load a file written by save_bin
    once, then predict initial weights for problems on their site lattice."""

    def __init__(self, path: str, device: int = 0):
        L = load()
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        L.cot_warmstart_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]
        L.cot_warmstart_free.argtypes = [vp]
        L.cot_warmstart_predict.argtypes = [vp, dp, dp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                            dp, dp, vp]
        L.cot_warmstart_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        self._L = L
        self._h = vp()
        rc = L.cot_warmstart_load(path.encode(), device, ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"cot_warmstart_load: {rc}: {self.error()}")

    @classmethod
    def from_npz(cls, npz_path: str, device: int = 0):
        """Load a network saved by np.savez(**WarmStartNet.state_dict()):
        written once more as the flat binary, then read through the C ABI."""
        import tempfile

        net = WarmStartNet.from_file(npz_path, device=f"cuda:{device}")
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "net.bin")
            net.save_bin(path)
            return cls(path, device)

    def error(self) -> str:
        buf = ctypes.create_string_buffer(512)
        self._L.cot_warmstart_last_error(buf, 512)
        return buf.value.decode()

    def predict(self, p) -> np.ndarray:
        dp = ctypes.POINTER(ctypes.c_double)
        gx, gy = p.grid
        xy = np.ascontiguousarray(p.xy, np.float64).reshape(-1)
        nu = np.ascontiguousarray(p.nu, np.float64)
        pic = np.ascontiguousarray(p.picture, np.float64)
        pd = np.ascontiguousarray(p.proj_domain, np.float64)
        out = np.zeros(p.n)
        rc = self._L.cot_warmstart_predict(self._h, xy.ctypes.data_as(dp), nu.ctypes.data_as(dp), gx, gy,
                                           pic.ctypes.data_as(dp), int(p.size[0]), int(p.size[1]),
                                           pd.ctypes.data_as(dp), out.ctypes.data_as(dp), None)
        if rc != 0:
            raise RuntimeError(f"cot_warmstart_predict: {rc}: {self.error()}")
        return out

    def close(self):
        if self._h:
            self._L.cot_warmstart_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# data, training, evaluation
# ---------------------------------------------------------------------------
def solve_pairs(probs, tol: float = 1e-5, history: int = 10, chunk: int = 64, method: str = "lbfgs"):
    """Converged weights of each problem (the training targets) to max-rel
    error tol: batched L-BFGS solves from w = 0 (capi.solve_batch), or with
    method="newton" the multilevel damped Newton pipeline
    (warm.WarmSolver), problem by problem."""
    from . import capi

    ws, stats = [], []
    if method == "newton":
        from .warm import WarmSolver

        with WarmSolver(start="multilevel", tol=tol, min_sites=1024) as ws_:
            for p in probs:
                w, st = ws_.solve(p)
                ws.append(w)
                stats.append(st)
        return ws, stats
    for k in range(0, len(probs), chunk):
        part = probs[k:k + chunk]
        sol = []
        for p in part:
            s = capi.Solver()
            s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
            sol.append(s)
        w, st = capi.solve_batch(sol, [np.zeros(p.n) for p in part], tol=tol, history=history, max_iter=100000)
        for s in sol:
            s.close()
        ws += w
        stats += st
    return ws, stats


def fit(net: WarmStartNet, X, Y, *, epochs: int = 30, batch: int = 16, lr: float = 1e-3, seed: int = 0,
        lam: float = 0.0, log=None) -> list:
    """Adam on the mean-free squared error.  X: bf16 [S, H, W, 8], Y: fp32
    [S, H*W] (device).  Returns the mean loss of every epoch."""
    torch = net.torch
    rng = np.random.default_rng(seed)
    S = X.shape[0]
    hist = []
    for ep in range(epochs):
        order = torch.from_numpy(rng.permutation(S)).to(X.device)
        tot, cnt = 0.0, 0
        for k in range(0, S - batch + 1, batch):
            idx = order[k:k + batch]
            net.zero_grad()
            pred = net.forward(X.index_select(0, idx), keep=True)
            loss, g = net.loss_grad(pred, Y.index_select(0, idx), grid=tuple(X.shape[1:3]), lam=lam)
            net.backward(g)
            net.adam(lr=lr)
            tot += loss
            cnt += 1
        hist.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return hist


def compare(net: WarmStartNet, probs, *, tol: float = 1e-4, history: int = 10, chunk: int = 64):
    """Cold (w = 0) and warm (network) solves of the same problems to max-rel
    error tol, each arm as batched solves.  Returns a dict of per-instance
    iterations and evaluations, the final errors and the device seconds of
    each arm (the warm arm includes the network's inference)."""
    import time

    from . import capi

    torch = net.torch
    out = {"cold_iters": [], "warm_iters": [], "cold_evals": [], "warm_evals": [], "cold_err": [], "warm_err": [],
           "cold_s": 0.0, "warm_s": 0.0, "infer_s": 0.0}
    for k in range(0, len(probs), chunk):
        part = probs[k:k + chunk]
        for arm in ("cold", "warm"):
            sol = []
            for p in part:
                s = capi.Solver()
                s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
                sol.append(s)
            if arm == "warm":
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                w0 = predict(net, part)
                torch.cuda.synchronize()
                out["infer_s"] += time.perf_counter() - t0
            else:
                w0 = [np.zeros(p.n) for p in part]
            _, st = capi.solve_batch(sol, w0, tol=tol, history=history, max_iter=100000)
            for s in sol:
                s.close()
            out[f"{arm}_iters"] += [x.iterations for x in st]
            out[f"{arm}_evals"] += [x.evaluations for x in st]
            out[f"{arm}_err"] += [x.max_rel_err for x in st]
            out[f"{arm}_s"] += st[0].ms * 1e-3
    out["warm_s"] += out["infer_s"]
    return out


def main(argv=None) -> int:
    """Generate solver-made pairs of the warm-start configuration (128x128
    jittered sites, 256^2 Gaussian-mixture targets, weights converged to
    1e-5), train the network, save it, and compare warm and cold solves of
    held-out seeds to 1e-4.  Prints one JSON line."""
    import argparse
    import json
    import time

    import torch

    from . import problems

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--held", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lam", type=float, default=0.0, help="weight of the neighbour-difference term of the loss")
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--base", type=int, default=32)
    ap.add_argument("--grid", type=int, default=0, help="sites per side (0: the configuration's 128)")
    ap.add_argument("--res", type=int, default=0, help="image pixels per side (0: the configuration's 256)")
    ap.add_argument("--config", type=int, default=4,
                    help="problem generator: 4 (uniform masses, K in 2..16) or 2 (beam masses, K = 16)")
    ap.add_argument("--uniform-fraction", type=float, default=0.0,
                    help="with --config 2: share of the pairs drawn with uniform masses instead of the beam")
    ap.add_argument("--solver", choices=["lbfgs", "newton"], default="lbfgs",
                    help="how the training targets are solved")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    kw = {}
    if a.grid:
        kw["g"] = a.grid
    if a.res:
        kw["res"] = a.res
    t0 = time.perf_counter()

    def make(i):
        if a.config == 2 and a.uniform_fraction > 0 and (i * 0.6180339887) % 1.0 < a.uniform_fraction:
            return problems.make(2, i, beam=False, **kw)
        return problems.make(a.config, i, **kw)

    train = [make(i) for i in range(a.pairs)]
    held = [make(100000 + i) for i in range(a.held)]
    ws, st = solve_pairs(train, tol=1e-5, method=a.solver)
    t_data = time.perf_counter() - t0
    net = WarmStartNet(levels=a.levels, base=a.base, seed=0)
    X = make_input(train)
    Y, net.out_scale = make_target(ws)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = fit(net, X, Y, epochs=a.epochs, batch=a.batch, lr=a.lr, lam=a.lam)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    if a.out:
        np.savez(a.out, **net.state_dict())
    res = compare(net, held, tol=1e-4)
    line = {"pairs": a.pairs, "held": a.held, "n_sites": train[0].n, "image": list(train[0].size), "lam": a.lam,
            "data_s": t_data, "pairs_converged": int(sum(s.converged for s in st)),
            "train_s": t_train, "epochs": a.epochs, "loss_first": hist[0], "loss_last": hist[-1],
            "cold_iters_mean": float(np.mean(res["cold_iters"])), "warm_iters_mean": float(np.mean(res["warm_iters"])),
            "cold_evals_mean": float(np.mean(res["cold_evals"])), "warm_evals_mean": float(np.mean(res["warm_evals"])),
            "cold_s": res["cold_s"], "warm_s": res["warm_s"], "infer_s": res["infer_s"],
            "cold_max_err": float(max(res["cold_err"])), "warm_max_err": float(max(res["warm_err"]))}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
