"""The learned-guess U-Net on the GPU (tensor-core convolutions, BF16
activations) against its FP32 numpy restatement (tests/nn_oracle.py): output,
loss and every parameter gradient.  Tolerances cover BF16 rounding of the
activations and activation gradients at every layer: 3e-2 of the output's
max norm, 0.1 relative L2 per gradient tensor."""
import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import learned as LN
from tests import nn_oracle as NO

pytestmark = pytest.mark.gpu

DIMS = (8, 16, 64)


@pytest.fixture(scope="module")
def net(tmp_path_factory):
    from artss_b200 import scenes
    sc = scenes.plume_box(n=16, steps=1, n_level=1)
    ctx = A.Context(A.Geometry(scenes.write(sc, str(tmp_path_factory.mktemp("u") / "b.xml"))))
    yield ctx, LN.UNet(ctx, DIMS, seed=3)
    ctx.close()


def to_dev(buf, a):
    import torch
    buf.copy_(torch.from_numpy(LN.to_bf16_bits(a).view(np.int16).ravel()).view(torch.bfloat16))
    torch.cuda.synchronize()


def params(u):
    return {name: (getattr(u, name).w.cpu().numpy(), getattr(u, name).b.cpu().numpy()) for name in NO.ORDER}


def test_unet_forward_backward(net):
    import torch
    ctx, u = net
    D, H, W = DIMS
    rng = np.random.default_rng(0)
    x = np.zeros((D, H, W, 16), np.float32)
    mask = (rng.random((D, H, W)) > 0.1).astype(np.float32)
    x[..., 0] = rng.standard_normal((D, H, W)) * mask
    x[..., 1] = mask
    x[..., 2] = rng.standard_normal((D, H, W)) * mask
    x = LN.round_bf16(x)
    target = (rng.standard_normal((D, H, W)) * 0.1).astype(np.float32)
    to_dev(u.buf["x"], x)
    t_dev = torch.from_numpy(target.ravel()).cuda()
    torch.cuda.synchronize()
    out = u.forward()
    loss = u.loss_grad(t_dev, int(mask.sum()))
    u.backward()
    A.cuda_check(u.lib.artss_nn_check(u.h), "network")
    ref_loss, ref_g, ref_a = NO.loss_and_grads(params(u), x, target, mask)
    got = out.float().cpu().numpy().reshape(D, H, W, 16)[..., 0]
    ref = ref_a["out"][..., 0]
    assert np.abs(got - ref).max() <= 3e-2 * np.abs(ref).max()
    assert abs(loss - ref_loss) <= 3e-2 * ref_loss
    for name in NO.ORDER:
        layer = getattr(u, name)
        for g_dev, g_ref in zip(layer.grads, ref_g[name]):
            g = g_dev.cpu().numpy().reshape(g_ref.shape)
            err = np.linalg.norm(g - g_ref) / max(np.linalg.norm(g_ref), 1e-30)
            assert err <= 0.1, (name, err)


def test_unet_adam_reduces_loss(net):
    import torch
    ctx, u = net
    D, H, W = DIMS
    rng = np.random.default_rng(1)
    x = np.zeros((D, H, W, 16), np.float32)
    x[..., 0] = rng.standard_normal((D, H, W))
    x[..., 1] = 1.0
    x = LN.round_bf16(x)
    # a target the network can fit: a smooth function of the input
    target = (0.3 * x[..., 0]).astype(np.float32)
    to_dev(u.buf["x"], x)
    t_dev = torch.from_numpy(target.ravel()).cuda()
    losses = []
    for _ in range(30):
        u.forward()
        losses.append(u.loss_grad(t_dev, D * H * W))
        u.backward()
        u.adam(lr=3e-3)
    assert losses[-1] < 0.5 * losses[0], losses
