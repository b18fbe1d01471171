"""Learned initial guess of the pressure solve: a small 3-D U-Net whose
convolutions run on the tensor cores (include/artss_cuda.h, artss_conv3d_*).
No counterpart in the reference.

Host-side helpers: BF16 conversion and the weight packing the convolution
kernels expect.  Device buffers are torch tensors used as plain memory; every
operation on them is a kernel of libartss_cuda.so."""
from __future__ import annotations

import numpy as np


def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.ascontiguousarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def round_bf16(a: np.ndarray) -> np.ndarray:
    return from_bf16_bits(to_bf16_bits(a))


def pack_conv_weights(w: np.ndarray) -> np.ndarray:
    """w[co][ci][kz][ky][kx] -> [27][ci/8][co][8] (tap t = 9 kz + 3 ky + kx),
    the per-tap shared-memory layout of the convolution's B operand."""
    co, ci = w.shape[:2]
    assert w.shape[2:] == (3, 3, 3) and ci % 8 == 0
    t = np.ascontiguousarray(w.reshape(co, ci, 27).transpose(2, 1, 0))  # [27][ci][co]
    return np.ascontiguousarray(t.reshape(27, ci // 8, 8, co).transpose(0, 1, 3, 2))  # [27][ci/8][co][8]


def conv3d_ref(x: np.ndarray, w: np.ndarray, bias=None, relu=False) -> np.ndarray:
    """FP32 reference: x[D][H][W][ci], w[co][ci][3][3][3], zero padding 1."""
    D, H, W, ci = x.shape
    co = w.shape[0]
    xp = np.zeros((D + 2, H + 2, W + 2, ci), np.float32)
    xp[1:-1, 1:-1, 1:-1] = x
    y = np.zeros((D, H, W, co), np.float32)
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                y += np.einsum("zyxc,oc->zyxo", xp[kz:kz + D, ky:ky + H, kx:kx + W], w[:, :, kz, ky, kx],
                               optimize=True)
    if bias is not None:
        y += bias
    if relu:
        y = np.maximum(y, 0)
    return y


def flip_weights(w: np.ndarray) -> np.ndarray:
    """Weights of the input-gradient convolution: w'[ci][co][t] = w[co][ci][26 - t]."""
    return np.ascontiguousarray(w.transpose(1, 0, 2, 3, 4)[:, :, ::-1, ::-1, ::-1])


def conv3d_wgrad_ref(x: np.ndarray, dy: np.ndarray) -> np.ndarray:
    """FP32 reference: dw[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci]."""
    D, H, W, ci = x.shape
    co = dy.shape[3]
    xp = np.zeros((D + 2, H + 2, W + 2, ci), np.float32)
    xp[1:-1, 1:-1, 1:-1] = x
    dw = np.zeros((27, co, ci), np.float32)
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                dw[9 * kz + 3 * ky + kx] = np.einsum("zyxo,zyxc->oc", dy, xp[kz:kz + D, ky:ky + H, kx:kx + W],
                                                     optimize=True)
    return dw


# ---------------------------------------------------------------- the network
import ctypes as _C


def _p(t):
    return _C.c_void_p(t.data_ptr())


class Conv:
    """One 3x3x3 convolution (+ bias, optional ReLU) with FP32 master weights
    w[27][cout][cin], their BF16 packed operands, gradients and Adam moments."""

    def __init__(self, net, cin: int, cout: int, relu: bool, rng, cin_real: int = None):
        import torch
        self.net, self.cin, self.cout, self.relu = net, cin, cout, relu
        ci = cin_real or cin
        w = np.zeros((27, cout, cin), np.float32)
        w[:, :, :ci] = rng.standard_normal((27, cout, ci)) * np.sqrt(2.0 / (27 * ci))
        dev = net.device
        self.w = torch.from_numpy(w).to(dev)
        self.b = torch.zeros(cout, dtype=torch.float32, device=dev)
        self.params = [self.w, self.b]
        self.grads = [torch.empty_like(self.w), torch.empty_like(self.b)]
        self.m = [torch.zeros_like(self.w), torch.zeros_like(self.b)]
        self.v = [torch.zeros_like(self.w), torch.zeros_like(self.b)]
        self.pw = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=dev)
        self.pf = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=dev)

    def pack(self):
        L, h = self.net.lib, self.net.h
        _ck(L.artss_nn_pack_weights(h, _p(self.w), _p(self.pw), self.cout, self.cin, 0), "pack")
        _ck(L.artss_nn_pack_weights(h, _p(self.w), _p(self.pf), self.cout, self.cin, 1), "pack flip")

    def desc(self, dims, cin, cout, relu):
        from artss_b200 import ConvDesc
        return ConvDesc(dims[0], dims[1], dims[2], cin, cout, int(relu))

    def fwd(self, x, y, dims):
        d = self.desc(dims, self.cin, self.cout, self.relu)
        _ck(self.net.lib.artss_conv3d_fwd(self.net.h, _C.byref(d), _p(x), _p(self.pw), _p(self.b), _p(y)), "conv")

    def bwd(self, x, y, dy, dx, dims):
        """dy: gradient of this layer's output (modified in place by the ReLU
        mask); accumulates the parameter gradients; dx (or None) receives the
        gradient of the input."""
        L, h = self.net.lib, self.net.h
        vox = dims[0] * dims[1] * dims[2]
        if self.relu:
            _ck(L.artss_nn_relu_bwd(h, _p(dy), _p(y), vox * self.cout), "relu bwd")
        _ck(L.artss_nn_bias_grad(h, _p(dy), _p(self.grads[1]), vox, self.cout), "bias grad")
        d = self.desc(dims, self.cin, self.cout, 0)
        _ck(L.artss_conv3d_wgrad(h, _C.byref(d), _p(x), _p(dy), _p(self.grads[0])), "wgrad")
        if dx is not None:
            db = self.desc(dims, self.cout, self.cin, 0)
            _ck(L.artss_conv3d_fwd(h, _C.byref(db), _p(dy), _p(self.pf), None, _p(dx)), "dgrad")


def _ck(status, what):
    from artss_b200 import cuda_check
    cuda_check(status, what)


class UNet:
    """3-level 3-D U-Net (channels 16-32-64, 3x3x3 convolutions, BF16
    activations, FP32 accumulation and parameters) mapping (rhs, obstacle
    mask, previous pressure) to a pressure correction; every operation is a
    kernel of libartss_cuda.so on the context's stream.

        x(16) -c-> a0(16) -c-> s0(16) -pool-> p0(16) -c-> a1(32) -c-> s1(32)
        -pool-> p1(32) -c-> a2(64) -c-> b2(64) -up, cat s1-> cat1(96) -c-> e1(32)
        -c-> d1(32) -up, cat s0-> cat0(48) -c-> e0(16) -c-> out(16, ch 0 used)
    """

    C_IN = 16

    def __init__(self, ctx, dims, seed: int = 0):
        import torch
        from artss_b200 import load_cuda
        self.ctx, self.h, self.lib = ctx, ctx.h, load_cuda()
        self.device = torch.device("cuda", torch.cuda.current_device())
        D, H, W = dims
        assert D % 4 == 0 and H % 4 == 0 and W % 4 == 0
        self.dims = [(D, H, W), (D // 2, H // 2, W // 2), (D // 4, H // 4, W // 4)]
        rng = np.random.default_rng(seed)
        self.e0a = Conv(self, 16, 16, True, rng, cin_real=3)
        self.e0b = Conv(self, 16, 16, True, rng)
        self.e1a = Conv(self, 16, 32, True, rng)
        self.e1b = Conv(self, 32, 32, True, rng)
        self.b2a = Conv(self, 32, 64, True, rng)
        self.b2b = Conv(self, 64, 64, True, rng)
        self.d1a = Conv(self, 96, 32, True, rng)
        self.d1b = Conv(self, 32, 32, True, rng)
        self.d0a = Conv(self, 48, 16, True, rng)
        self.d0b = Conv(self, 16, 16, False, rng)
        self.layers = [self.e0a, self.e0b, self.e1a, self.e1b, self.b2a, self.b2b, self.d1a, self.d1b, self.d0a,
                       self.d0b]
        sizes = {"x": (0, 16), "a0": (0, 16), "s0": (0, 16), "p0": (1, 16), "a1": (1, 32), "s1": (1, 32),
                 "p1": (2, 32), "a2": (2, 64), "b2": (2, 64), "cat1": (1, 96), "e1": (1, 32), "d1": (1, 32),
                 "cat0": (0, 48), "e0": (0, 16), "out": (0, 16)}
        self.buf = {k: self._act(l, c) for k, (l, c) in sizes.items()}
        gs = {"out": (0, 16), "e0": (0, 16), "cat0": (0, 48), "s0": (0, 16), "t0": (0, 16), "a0": (0, 16),
              "d1": (1, 32), "e1": (1, 32), "cat1": (1, 96), "s1": (1, 32), "t1": (1, 32), "p0": (1, 16),
              "a1": (1, 32), "b2": (2, 64), "a2": (2, 64), "p1": (2, 32)}
        self.grad = {k: self._act(l, c) for k, (l, c) in gs.items()}
        self.step_no = 0
        self.pack()

    def _act(self, level, c):
        import torch
        D, H, W = self.dims[level]
        return torch.empty(D * H * W * c, dtype=torch.bfloat16, device=self.device)

    def vox(self, level):
        D, H, W = self.dims[level]
        return D * H * W

    def pack(self):
        for l in self.layers:
            l.pack()

    def forward(self):
        """Runs the network on buf['x'] ([D][H][W][16] bf16); returns buf['out']."""
        B, L, h, d = self.buf, self.lib, self.h, self.dims
        self.e0a.fwd(B["x"], B["a0"], d[0])
        self.e0b.fwd(B["a0"], B["s0"], d[0])
        _ck(L.artss_nn_pool2(h, _p(B["s0"]), _p(B["p0"]), *d[0], 16, 0), "pool")
        self.e1a.fwd(B["p0"], B["a1"], d[1])
        self.e1b.fwd(B["a1"], B["s1"], d[1])
        _ck(L.artss_nn_pool2(h, _p(B["s1"]), _p(B["p1"]), *d[1], 32, 0), "pool")
        self.b2a.fwd(B["p1"], B["a2"], d[2])
        self.b2b.fwd(B["a2"], B["b2"], d[2])
        _ck(L.artss_nn_up2(h, _p(B["b2"]), _p(B["cat1"]), *d[2], 64, 96, 0, 0), "up")
        _ck(L.artss_nn_copy_channels(h, _p(B["s1"]), 32, 0, _p(B["cat1"]), 96, 64, 32, self.vox(1), 0), "cat")
        self.d1a.fwd(B["cat1"], B["e1"], d[1])
        self.d1b.fwd(B["e1"], B["d1"], d[1])
        _ck(L.artss_nn_up2(h, _p(B["d1"]), _p(B["cat0"]), *d[1], 32, 48, 0, 0), "up")
        _ck(L.artss_nn_copy_channels(h, _p(B["s0"]), 16, 0, _p(B["cat0"]), 48, 32, 16, self.vox(0), 0), "cat")
        self.d0a.fwd(B["cat0"], B["e0"], d[0])
        self.d0b.fwd(B["e0"], B["out"], d[0])
        return B["out"]

    def backward(self):
        """Gradients of every parameter from grad['out'] (set by the loss)."""
        B, G, L, h, d = self.buf, self.grad, self.lib, self.h, self.dims
        for l in self.layers:
            for g in l.grads:
                _ck(L.artss_nn_zero(h, _p(g), g.numel() * 4), "zero")
        self.d0b.bwd(B["e0"], B["out"], G["out"], G["e0"], d[0])
        self.d0a.bwd(B["cat0"], B["e0"], G["e0"], G["cat0"], d[0])
        _ck(L.artss_nn_up2(h, _p(G["cat0"]), _p(G["d1"]), *d[1], 32, 48, 0, 1), "up bwd")
        _ck(L.artss_nn_copy_channels(h, _p(G["cat0"]), 48, 32, _p(G["s0"]), 16, 0, 16, self.vox(0), 0), "split")
        self.d1b.bwd(B["e1"], B["d1"], G["d1"], G["e1"], d[1])
        self.d1a.bwd(B["cat1"], B["e1"], G["e1"], G["cat1"], d[1])
        _ck(L.artss_nn_up2(h, _p(G["cat1"]), _p(G["b2"]), *d[2], 64, 96, 0, 1), "up bwd")
        _ck(L.artss_nn_copy_channels(h, _p(G["cat1"]), 96, 64, _p(G["s1"]), 32, 0, 32, self.vox(1), 0), "split")
        self.b2b.bwd(B["a2"], B["b2"], G["b2"], G["a2"], d[2])
        self.b2a.bwd(B["p1"], B["a2"], G["a2"], G["p1"], d[2])
        _ck(L.artss_nn_pool2(h, _p(G["p1"]), _p(G["t1"]), *d[1], 32, 1), "pool bwd")
        _ck(L.artss_nn_copy_channels(h, _p(G["t1"]), 32, 0, _p(G["s1"]), 32, 0, 32, self.vox(1), 1), "add")
        self.e1b.bwd(B["a1"], B["s1"], G["s1"], G["a1"], d[1])
        self.e1a.bwd(B["p0"], B["a1"], G["a1"], G["p0"], d[1])
        _ck(L.artss_nn_pool2(h, _p(G["p0"]), _p(G["t0"]), *d[0], 16, 1), "pool bwd")
        _ck(L.artss_nn_copy_channels(h, _p(G["t0"]), 16, 0, _p(G["s0"]), 16, 0, 16, self.vox(0), 1), "add")
        self.e0b.bwd(B["a0"], B["s0"], G["s0"], G["a0"], d[0])
        self.e0a.bwd(B["x"], B["a0"], G["a0"], None, d[0])

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_no += 1
        for l in self.layers:
            for p, g, m, v in zip(l.params, l.grads, l.m, l.v):
                _ck(self.lib.artss_nn_adam(self.h, _p(p), _p(g), _p(m), _p(v), p.numel(), lr, b1, b2, eps,
                                           self.step_no), "adam")
        self.pack()

    def loss_grad(self, target, n_fluid: int):
        """0.5 mean over fluid voxels of (out[.][0] - target)^2; sets grad['out']."""
        import torch
        nb = 296
        part = torch.empty(nb, dtype=torch.float32, device=self.device)
        _ck(self.lib.artss_nn_mse(self.h, _p(self.buf["out"]), 16, _p(target), _p(self.buf["x"]),
                                  _p(self.grad["out"]), self.vox(0), 1.0 / max(n_fluid, 1), _p(part), nb), "mse")
        _ck(self.lib.artss_nn_check(self.h), "network")
        return float(part.cpu().numpy().astype(np.float64).sum()) / max(n_fluid, 1)
