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
