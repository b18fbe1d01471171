"""The learned initial guess end to end on a small channel: training samples
from the solver, training on the GPU by the network's own kernels, and the
evaluation against the previous-pressure start and against the plain FP64
VCycleMG.  The guess is p_prev + alpha * correction with alpha minimising the
residual over the line (learned.min_residual_step), so its initial residual
is never above the previous pressure's: the network can only help."""
import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import learned as LN

pytestmark = pytest.mark.gpu

DIMS = (32, 32, 64)


def test_learned_guess_pipeline(tmp_path):
    samples = LN.collect([11, 12], 4, 5, DIMS, str(tmp_path), project=2)
    assert len(samples) == 8 and all(s["cycles"] > 0 for s in samples)
    sc = LN.plume_channel(0, nx=DIMS[2], ny=DIMS[1], nz=DIMS[0])
    from artss_b200 import scenes
    sim = A.Simulation(scenes.write(sc, str(tmp_path / "net.xml")))
    try:
        net = LN.UNet(sim.context, DIMS, seed=0)
        hist = LN.train(net, samples, epochs=3, lr=1e-3)
        assert np.isfinite(hist).all() and hist[-1] < hist[0]
        res = LN.evaluate(net, [21], 3, 5, DIMS, str(tmp_path), project=2, with_plain=True)
    finally:
        sim.close()
    n = len(res["baseline_cycles"])
    assert n == 3 and len(res["learned_cycles"]) == n and len(res["plain_cycles"]) == n
    # the minimal-residual step never raises the initial residual (up to
    # rounding), so no guess is discarded and no solve needs more than one
    # extra cycle than the previous-pressure start
    assert len(res["alpha"]) == n and all(np.isfinite(res["alpha"]))
    for lc, bc, ratio in zip(res["learned_cycles"], res["baseline_cycles"], res["residual_ratio"]):
        assert 0 < ratio <= 1 + 1e-9
        assert lc <= bc + 1
    assert res["fallbacks"] == 0
    print("learned guess: residual ratios", [round(r, 4) for r in res["residual_ratio"]], "alpha",
          [round(a, 4) for a in res["alpha"]], "cycles", res["learned_cycles"], "vs", res["baseline_cycles"])
    # the mixed-precision solve needs no more cycles than the plain FP64 V-cycle
    assert sum(res["baseline_cycles"]) <= sum(res["plain_cycles"])
