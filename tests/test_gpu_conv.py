"""BF16 tensor-core 3-D convolution (artss_conv3d_fwd) against an FP32 numpy
convolution of the same BF16-rounded inputs; tolerance: BF16 output rounding
plus FP32 accumulation-order differences, 1e-2 of the output's max norm."""
import ctypes as C

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import learned as LN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(tmp_path_factory):
    from artss_b200 import scenes
    sc = scenes.plume_box(n=16, steps=1, n_level=1)
    c = A.Context(A.Geometry(scenes.write(sc, str(tmp_path_factory.mktemp("c") / "b.xml"))))
    yield c
    c.close()


def dev_bf16(a):
    import torch
    return torch.from_numpy(LN.to_bf16_bits(a).view(np.int16)).view(torch.bfloat16).cuda()


@pytest.mark.parametrize("shape,cin,cout,relu", [
    ((4, 8, 32), 16, 16, 0),
    ((4, 8, 32), 32, 64, 1),
    ((3, 4, 64), 48, 32, 1),
    ((2, 2, 128), 16, 16, 0),
    ((8, 4, 16), 32, 16, 1),
])
def test_conv3d_fwd(ctx, shape, cin, cout, relu):
    import torch
    D, H, W = shape
    rng = np.random.default_rng(cin * 7 + cout)
    x = LN.round_bf16(rng.standard_normal((D, H, W, cin)).astype(np.float32))
    w = LN.round_bf16((rng.standard_normal((cout, cin, 3, 3, 3)) / np.sqrt(27 * cin)).astype(np.float32))
    bias = rng.standard_normal(cout).astype(np.float32) * 0.1
    ref = LN.conv3d_ref(x, w, bias, bool(relu))
    dx = dev_bf16(x)
    dw = dev_bf16(LN.pack_conv_weights(w))
    db = torch.from_numpy(bias).cuda()
    dy = torch.zeros((D, H, W, cout), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    d = A.ConvDesc(D, H, W, cin, cout, relu)
    A.cuda_check(ctx.lib.artss_conv3d_fwd(ctx.h, C.byref(d), dx.data_ptr(), dw.data_ptr(), db.data_ptr(),
                                          dy.data_ptr()), "conv")
    A.cuda_check(ctx.lib.artss_nn_check(ctx.h), "conv wait")
    got = dy.float().cpu().numpy()
    err = np.abs(got - ref).max()
    assert err <= 1e-2 * np.abs(ref).max() + 1e-6, err


@pytest.mark.parametrize("shape,cin,cout", [((4, 8, 32), 16, 32), ((2, 2, 128), 32, 16)])
def test_conv3d_input_grad(ctx, shape, cin, cout):
    """dX = the forward convolution of dY with flipped, transposed weights."""
    import torch
    D, H, W = shape
    rng = np.random.default_rng(3 * cin + cout)
    w = LN.round_bf16((rng.standard_normal((cout, cin, 3, 3, 3)) / np.sqrt(27 * cout)).astype(np.float32))
    dy = LN.round_bf16(rng.standard_normal((D, H, W, cout)).astype(np.float32))
    wf = LN.flip_weights(w)
    ref = LN.conv3d_ref(dy, wf)
    # the same as the adjoint of the forward map: <conv(x), dy> = <x, dx>
    x = rng.standard_normal((D, H, W, cin)).astype(np.float32)
    assert abs(np.vdot(LN.conv3d_ref(x, w), dy) - np.vdot(x, ref)) <= 1e-3 * abs(np.vdot(x, ref)) + 1e-3
    ddy, dwf = dev_bf16(dy), dev_bf16(LN.pack_conv_weights(wf))
    dx = torch.zeros((D, H, W, cin), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    d = A.ConvDesc(D, H, W, cout, cin, 0)
    A.cuda_check(ctx.lib.artss_conv3d_fwd(ctx.h, C.byref(d), ddy.data_ptr(), dwf.data_ptr(), None, dx.data_ptr()),
                 "conv dgrad")
    A.cuda_check(ctx.lib.artss_nn_check(ctx.h), "wait")
    got = dx.float().cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-2 * np.abs(ref).max()


@pytest.mark.parametrize("shape,cin,cout", [((4, 8, 32), 16, 32), ((2, 4, 64), 32, 16), ((2, 2, 128), 16, 64),
                                            ((4, 4, 16), 96, 32)])
def test_conv3d_weight_grad(ctx, shape, cin, cout):
    import torch
    D, H, W = shape
    rng = np.random.default_rng(5 * cin + cout)
    x = LN.round_bf16(rng.standard_normal((D, H, W, cin)).astype(np.float32))
    dy = LN.round_bf16(rng.standard_normal((D, H, W, cout)).astype(np.float32))
    ref = LN.conv3d_wgrad_ref(x, dy)
    dx_, ddy = dev_bf16(x), dev_bf16(dy)
    dw = torch.zeros((27, cout, cin), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    d = A.ConvDesc(D, H, W, cin, cout, 0)
    for _ in range(2):  # accumulates
        A.cuda_check(ctx.lib.artss_conv3d_wgrad(ctx.h, C.byref(d), dx_.data_ptr(), ddy.data_ptr(), dw.data_ptr()),
                     "wgrad")
    A.cuda_check(ctx.lib.artss_nn_check(ctx.h), "wait")
    got = dw.cpu().numpy()
    assert np.abs(got - 2 * ref).max() <= 1e-4 * np.abs(ref).max() + 1e-4
