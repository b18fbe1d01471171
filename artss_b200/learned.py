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
        """ctx: an artss_b200.Context or a raw artss_ctx handle (the network's
        kernels run on that context's stream)."""
        import torch
        from artss_b200 import load_cuda
        self.ctx, self.lib = ctx, load_cuda()
        self.h = ctx.h if hasattr(ctx, "h") else ctx
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

    def forward(self, x=None):
        """Runs the network on x ([D][H][W][16] bf16; default buf['x']);
        returns buf['out'].  backward() and loss_grad() use the same x."""
        B, L, h, d = self.buf, self.lib, self.h, self.dims
        self.x = B["x"] if x is None else x
        self.e0a.fwd(self.x, B["a0"], d[0])
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
        self.e0a.bwd(self.x, B["a0"], G["a0"], None, d[0])

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
        _ck(self.lib.artss_nn_mse(self.h, _p(self.buf["out"]), 16, _p(target), _p(self.x),
                                  _p(self.grad["out"]), self.vox(0), 1.0 / max(n_fluid, 1), _p(part), nb), "mse")
        _ck(self.lib.artss_nn_check(self.h), "network")
        return float(part.cpu().numpy().astype(np.float64).sum()) / max(n_fluid, 1)


# ------------------------------------------------------- data, training, use
def plume_channel(seed: int, nx: int = 128, ny: int = 64, nz: int = 64, steps: int = 10 ** 6):
    """A seeded scene of the ensemble family: the 6.4 x 3.2 x 3.2 m channel with
    an open (Dirichlet p) outflow, inflow U[0.2, 1.0] m/s, a Gaussian source of
    U[10, 150] kW centred at U[0.2, 0.8] of the extent, 0-3 box obstacles with
    edges of 2-8 coarse cells.  The open outflow keeps the pressure problem
    non-singular, so every right-hand side is solvable to any tolerance."""
    import random
    from artss_b200 import scenes
    rng = random.Random(7919 * seed + 1)
    sc = scenes.channel_with_cube(nx=nx, ny=ny, nz=nz, steps=steps, n_level=4)
    u_in = rng.uniform(0.2, 1.0)
    sc.boundaries = [b if not (b[0] == "u" and b[1] == "left") else ("u", "left", "dirichlet", u_in)
                     for b in sc.boundaries]
    sc.hrr = rng.uniform(10.0, 150.0)
    ext = (sc.X[1] - sc.X[0], sc.Y[1] - sc.Y[0], sc.Z[1] - sc.Z[0])
    sc.source_pos = tuple(lo + rng.uniform(0.2, 0.8) * e for lo, e in zip((sc.X[0], sc.Y[0], sc.Z[0]), ext))
    h = (ext[0] / nx, ext[1] / ny, ext[2] / nz)
    sc.obstacles = scenes.random_boxes((nx, ny, nz), 2 * 8, 8 * 8, rng.randint(0, 3), seed, h,
                                       origin=(sc.X[0], sc.Y[0], sc.Z[0]), levels=3)
    sc.seed = seed
    return sc


class Sampler:
    """Pressure problems of a running simulation: each sample() advances the
    scene by one timestep and records (rhs, mask, p_prev) -> p_star, where
    p_prev is the pressure before the step and p_star the step's pressure
    equation solved to `rel_tol` from p_prev by the mixed-precision solver.
    Inputs and targets are stored on the device in the network's layout."""

    def __init__(self, sim, dims, h: float, rel_tol: float = 1e-8, n_level: int = 4, project: int = 0):
        import torch
        from artss_b200 import MixedCfg, load_cuda
        self.sim, self.ctx, self.lib = sim, sim.context, load_cuda()
        self.dims = dims
        self.vox = dims[0] * dims[1] * dims[2]
        self.size = sim.size
        self.p_prev = self._field()
        self.p_star = self._field()
        self.zero = self._field()
        self.diff = self._field()
        self.project = project
        _ck(self.lib.artss_fill(self.ctx, self.zero, 0, 0.0), "fill")
        cfg = MixedCfg(n_level, 2, 1, 0, 0.6666666667, 0.0, 1e-3, 40, rel_tol, 200)
        self.mx = _C.c_void_p()
        _ck(self.lib.artss_mixed_create(self.ctx, _C.byref(cfg), _C.byref(self.mx)), "mixed")
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.rel_tol = rel_tol
        ext = min(dims) * h  # shortest domain extent (cell size h, isotropic grid)
        self.c = ext * ext / (np.pi * np.pi)

    def _field(self):
        from artss_b200 import _D
        p = _D()
        _ck(self.lib.artss_field_alloc(self.ctx, 0, _C.byref(p)), "alloc")
        return p

    def norm(self, f) -> float:
        r, bn = _C.c_double(), _C.c_double()
        _ck(self.lib.artss_residual_norm(self.ctx, self.zero, f, _C.byref(r), _C.byref(bn)), "norm")
        return bn.value

    def scales(self, rhs, p_prev):
        """(s_r, s_b, s_t): inputs scaled to unit RMS (the residual of p_prev and
        rhs) and the target's scale s_t = s_r / c, where c = L^2 / pi^2 for the
        shortest domain extent L converts a residual into a correction of the
        smoothest mode, A^-1 r ~ c r."""
        n = float(self.vox)
        r, bn = _C.c_double(), _C.c_double()
        _ck(self.lib.artss_apply_boundary(self.ctx, p_prev, 0, 4), "bc")
        _ck(self.lib.artss_residual_norm(self.ctx, p_prev, rhs, _C.byref(r), _C.byref(bn)), "norm")
        s_r = np.sqrt(n) / r.value if r.value > 0 else 1.0
        s_b = np.sqrt(n) / bn.value if bn.value > 0 else 1.0
        return s_r, s_b, s_r / self.c

    def inputs(self, rhs, p_prev, s_r, s_b, out):
        _ck(self.lib.artss_nn_inputs(self.ctx, 0, rhs, p_prev, s_r, s_b, _p(out), 16), "inputs")

    def solve(self, p, rhs):
        from artss_b200 import SolveStats
        st = SolveStats()
        _ck(self.lib.artss_mixed_solve(self.mx, p, rhs, _C.byref(st)), "solve")
        return st

    def sample(self):
        import torch
        from artss_b200 import _D
        p = _C.cast(_C.c_void_p(self.sim.device_pointer("p")), _D)
        rhs = _C.cast(_C.c_void_p(self.sim.device_pointer("rhs")), _D)
        _ck(self.lib.artss_copy(self.ctx, self.p_prev, p, 0), "copy")
        self.sim.run(1)
        _ck(self.lib.artss_copy(self.ctx, self.p_star, self.p_prev, 0), "copy")
        st = self.solve(self.p_star, rhs)
        s_r, s_b, s_t = self.scales(rhs, self.p_prev)
        x = torch.empty(self.vox * 16, dtype=torch.bfloat16, device=self.device)
        t = torch.empty(self.vox, dtype=torch.float32, device=self.device)
        self.inputs(rhs, self.p_prev, s_r, s_b, x)
        if self.project:
            # target = the smooth part of p_star - p_prev (artss_coarse_project)
            _ck(self.lib.artss_scale_copy(self.ctx, self.diff, self.p_prev, -1.0, 0), "neg")
            _ck(self.lib.artss_add_field(self.ctx, self.diff, self.p_star, 0), "diff")
            _ck(self.lib.artss_coarse_project(self.ctx, self.diff, self.project), "project")
            _ck(self.lib.artss_nn_target(self.ctx, 0, self.diff, self.zero, s_t, _p(t)), "target")
        else:
            _ck(self.lib.artss_nn_target(self.ctx, 0, self.p_star, self.p_prev, s_t, _p(t)), "target")
        _ck(self.lib.artss_nn_check(self.ctx), "sample")
        return {"x": x, "t": t, "cycles": int(st.cycles), "n_fluid": int(self.sim.inner_cells)}

    def close(self):
        if self.mx:
            self.lib.artss_mixed_destroy(self.mx)
            self.mx = _C.c_void_p()
        for f in (self.p_prev, self.p_star, self.zero, self.diff):
            self.lib.artss_field_free(self.ctx, f)


def collect(seeds, per_scene: int, warmup: int, dims, tmpdir: str, device: int = 0, project: int = 0):
    """Training samples from the plain solver: per seeded scene, `warmup`
    timesteps, then `per_scene` sampled timesteps (see Sampler)."""
    import os
    from artss_b200 import Simulation, scenes
    out = []
    for seed in seeds:
        sc = plume_channel(seed, nx=dims[2], ny=dims[1], nz=dims[0])
        sim = Simulation(scenes.write(sc, os.path.join(tmpdir, f"train_{seed}.xml")), device=device)
        sim.run(warmup)
        smp = Sampler(sim, dims, (sc.X[1] - sc.X[0]) / sc.nx, project=project)
        for _ in range(per_scene):
            out.append(smp.sample())
        smp.close()
        sim.close()
    return out


def train(net: UNet, samples, epochs: int, lr: float = 1e-3, seed: int = 0):
    """Adam on 0.5 mean (prediction - target)^2 over fluid cells, one sample
    per step; returns the mean loss of every epoch."""
    rng = np.random.default_rng(seed)
    history = []
    for _ in range(epochs):
        tot = 0.0
        for i in rng.permutation(len(samples)):
            s = samples[i]
            net.forward(s["x"])
            tot += net.loss_grad(s["t"], s["n_fluid"])
            net.backward()
            net.adam(lr=lr)
        history.append(tot / max(len(samples), 1))
    return history


def min_residual_step(lib, ctx, guess, p_prev, d, rhs, zero) -> float:
    """guess = p_prev + alpha d with alpha minimising ||rhs - A guess||_2 over
    the inner cells: alpha = (r . A d) / (A d . A d), r = rhs - A p_prev, the
    dot product from three residual norms (polarisation identity; the pressure's
    boundary values are zero, so A is linear on d).  The guess's residual is
    never above the previous pressure's.  Returns alpha."""
    _ck(lib.artss_apply_boundary(ctx, d, 0, 4), "bc")
    ad, _ = _resnorm(lib, ctx, d, zero)             # ||A d||
    r0, _ = _resnorm(lib, ctx, p_prev, rhs)         # ||r||
    _ck(lib.artss_copy(ctx, guess, p_prev, 0), "copy")
    _ck(lib.artss_add_field(ctx, guess, d, 0), "add")
    _ck(lib.artss_apply_boundary(ctx, guess, 0, 4), "bc")
    r1, _ = _resnorm(lib, ctx, guess, rhs)          # ||r - A d||
    alpha = (r0 * r0 + ad * ad - r1 * r1) / (2.0 * ad * ad) if ad > 0 else 0.0
    _ck(lib.artss_copy(ctx, guess, p_prev, 0), "copy")
    if alpha != 0.0:
        _ck(lib.artss_scale(ctx, d, alpha, 0), "scale")
        _ck(lib.artss_add_field(ctx, guess, d, 0), "add")
    _ck(lib.artss_apply_boundary(ctx, guess, 0, 4), "bc")
    return alpha


def evaluate(net: UNet, seeds, steps: int, warmup: int, dims, tmpdir: str, device: int = 0, project: int = 2,
             with_plain: bool = False, min_residual: bool = True):
    """Per timestep of unseen scenes: the pressure equation solved to 1e-8 by
    the mixed-precision solver from (a) the previous pressure and (b) the
    network's guess p_prev + correction, the correction restricted `project`
    times and prolongated back (its smooth part; artss_coarse_project),
    falling back to (a) when the guess's initial residual is larger, and, with
    `with_plain`, (c) the plain FP64 VCycleMG from the previous pressure.
    Returns cycles and ms (CUDA events on the context stream; (b) includes the
    network's inference)."""
    import os
    import torch
    from artss_b200 import Simulation, SolveStats, _D, scenes
    res = {"baseline_cycles": [], "baseline_ms": [], "learned_cycles": [], "learned_ms": [], "fallbacks": 0,
           "infer_ms": [], "residual_ratio": [], "plain_cycles": [], "plain_ms": []}
    for seed in seeds:
        sc = plume_channel(seed, nx=dims[2], ny=dims[1], nz=dims[0])
        sim = Simulation(scenes.write(sc, os.path.join(tmpdir, f"eval_{seed}.xml")), device=device)
        sim.run(warmup)
        smp = Sampler(sim, dims, (sc.X[1] - sc.X[0]) / sc.nx)
        lib, ctx = smp.lib, smp.ctx
        stream = torch.cuda.ExternalStream(lib.artss_ctx_stream(ctx))
        guess, corr = smp._field(), smp._field()
        # L2 flush between timed solves: a buffer twice the 126 MB L2, zeroed on the stream
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=smp.device)

        def flush_l2():
            _ck(lib.artss_nn_zero(ctx, _p(flush), flush.numel()), "flush")
        plain = None
        if with_plain:
            from artss_b200 import MgCfg
            mc = MgCfg(sc.n_level, 2, 100, 2, 1e-8, 0, 0, 100, 1e-8, 0.6666666667)
            plain = _C.c_void_p()
            _ck(lib.artss_mg_create(ctx, _C.byref(mc), _C.byref(plain)), "plain")
        x = torch.empty(smp.vox * 16, dtype=torch.bfloat16, device=smp.device)
        for _ in range(steps):
            p = _C.cast(_C.c_void_p(sim.device_pointer("p")), _D)
            rhs = _C.cast(_C.c_void_p(sim.device_pointer("rhs")), _D)
            _ck(lib.artss_copy(ctx, smp.p_prev, p, 0), "copy")
            sim.run(1)
            # (a) from the previous pressure
            _ck(lib.artss_copy(ctx, smp.p_star, smp.p_prev, 0), "copy")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush_l2()
            e0.record(stream)
            st = smp.solve(smp.p_star, rhs)
            e1.record(stream)
            e1.synchronize()
            res["baseline_cycles"].append(int(st.cycles))
            res["baseline_ms"].append(e0.elapsed_time(e1))
            # (c) the plain FP64 VCycleMG from the previous pressure
            if plain is not None:
                _ck(lib.artss_copy(ctx, guess, smp.p_prev, 0), "copy")
                pst = SolveStats()
                flush_l2()
                e0.record(stream)
                _ck(lib.artss_mg_solve_rel(plain, guess, rhs, smp.rel_tol, 1000, _C.byref(pst)), "plain")
                e1.record(stream)
                e1.synchronize()
                res["plain_cycles"].append(int(pst.cycles))
                res["plain_ms"].append(e0.elapsed_time(e1))
            # (b) from the network's guess
            flush_l2()
            e0.record(stream)
            s_r, s_b, s_t = smp.scales(rhs, smp.p_prev)
            smp.inputs(rhs, smp.p_prev, s_r, s_b, x)
            out = net.forward(x)
            # correction = the network's output, kept to the coarse space of
            # `project` levels (its smooth part), added to p_prev
            _ck(lib.artss_fill(ctx, corr, 0, 0.0), "fill")
            _ck(lib.artss_nn_apply(ctx, 0, _p(out), 16, smp.zero, 1.0 / s_t, corr), "apply")
            if project:
                _ck(lib.artss_coarse_project(ctx, corr, project), "project")
            if min_residual:
                res.setdefault("alpha", []).append(min_residual_step(lib, ctx, guess, smp.p_prev, corr, rhs, smp.zero))
            else:
                _ck(lib.artss_copy(ctx, guess, smp.p_prev, 0), "copy")
                _ck(lib.artss_add_field(ctx, guess, corr, 0), "add")
                _ck(lib.artss_apply_boundary(ctx, guess, 0, 4), "bc")
            e2 = torch.cuda.Event(enable_timing=True)
            e2.record(stream)
            r_g, _ = _resnorm(lib, ctx, guess, rhs)
            r_p, _ = _resnorm(lib, ctx, smp.p_prev, rhs)
            res["residual_ratio"].append(r_g / r_p if r_p > 0 else 1.0)
            # (the minimal-residual step keeps r_g <= r_p up to rounding)
            if r_g > r_p * (1 + 1e-9):
                res["fallbacks"] += 1
                _ck(lib.artss_copy(ctx, guess, smp.p_prev, 0), "copy")
            st = smp.solve(guess, rhs)
            e1.record(stream)
            e1.synchronize()
            res["learned_cycles"].append(int(st.cycles))
            res["learned_ms"].append(e0.elapsed_time(e1))
            res["infer_ms"].append(e0.elapsed_time(e2))
        if plain is not None:
            lib.artss_mg_destroy(plain)
        lib.artss_field_free(ctx, guess)
        lib.artss_field_free(ctx, corr)
        smp.close()
        sim.close()
    return res


def _resnorm(lib, ctx, p, b):
    r, bn = _C.c_double(), _C.c_double()
    _ck(lib.artss_residual_norm(ctx, p, b, _C.byref(r), _C.byref(bn)), "residual")
    return r.value, bn.value
