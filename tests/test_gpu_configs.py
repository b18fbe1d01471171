"""Parity at the benchmarked sizes.

The small-scene parity tests (test_gpu_parity.py) cover every solver
composition; these two run the two plain-FP64 workloads themselves against
the reference serial build (oracle/_ref/artss_ref_driver):

* the 64^3 closed plume box (2.4 m, 4 multigrid levels, colored Gauss-Seidel
  diffusion, ConstSmagorinsky 0.2, 25 kW Gaussian source, dt 0.005 s) over
  200 steps, u, v, w, p, T and nu_t compared every 10 steps;
* the 256x128x128 channel with one cube that bench.py times (inflow
  0.5 m/s, 100 kW source, dt 0.002 s), steps 1-4 (step 1 iterates the
  pressure to tolerance), every field compared after every step, once with
  eager steps and once with whole-step graphs (the end-to-end path), plus the
  device cell flags against the reference's index lists at full size.

At these sizes the timed code paths run as in the benchmark: the TMA colored
Gauss-Seidel sweep at the autotuned depth, the pipelined cluster coarse solve
with its cross-rank boundary chains, the trimmed couples.  Bound: 1e-10
relative max-norm per field (the observed error is 0).
"""
import ctypes as C

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import refdriver

pytestmark = pytest.mark.gpu

TOL = 1e-10
FIELDS = ["u", "v", "w", "p", "T", "nu_t"]


def _need_ref():
    if not refdriver.available():
        pytest.skip("reference oracle not built (oracle/Makefile)")


def _compare(sim, dump, step, worst):
    for f in FIELDS:
        err = refdriver.rel_max_err(sim.field(f), refdriver.field(dump, step, f))
        worst[f] = max(worst[f], err)
        assert err <= TOL, f"step {step} field {f}: relative max error {err:.3e}"


def test_plume_box_64_200_steps(tmp_path):
    sc = scenes.plume_box()
    assert (sc.nx, sc.ny, sc.nz, sc.n_level, sc.steps, sc.dt) == (64, 64, 64, 4, 200, 0.005)
    _need_ref()
    xml = scenes.write(sc, str(tmp_path / "plume_box_64.xml"))
    dump = refdriver.run(xml, str(tmp_path / "ref"), steps=sc.steps, every=10, fields=FIELDS, timeout=1800)
    worst = {f: 0.0 for f in FIELDS}
    with A.Simulation(xml) as sim:
        _compare(sim, dump, 0, worst)
        for step in range(10, sc.steps + 1, 10):
            assert sim.run(10) == 10
            _compare(sim, dump, step, worst)
    print("plume box 64^3, 200 steps, worst relative error per field: " +
          ", ".join(f"{f} {e:.3e}" for f, e in worst.items()))


@pytest.fixture(scope="module")
def channel(tmp_path_factory):
    _need_ref()
    base = tmp_path_factory.mktemp("channel_full")
    sc = scenes.channel_with_cube(steps=4)
    assert (sc.nx, sc.ny, sc.nz, sc.n_level) == (256, 128, 128, 4)
    xml = scenes.write(sc, str(base / "channel_256x128x128.xml"))
    dump = refdriver.run(xml, str(base / "ref"), steps=4, every=1, lists=True, fields=FIELDS, timeout=1800)
    return xml, dump


@pytest.mark.parametrize("graphs", [False, True], ids=["eager", "graphs"])
def test_channel_256x128x128_steps_1_to_4(channel, graphs):
    xml, dump = channel
    worst = {f: 0.0 for f in FIELDS}
    with A.Simulation(xml) as sim:
        sim.set_graphs(graphs)
        _compare(sim, dump, 0, worst)
        for step in range(1, 5):
            assert sim.run(1) == 1
            _compare(sim, dump, step, worst)
        if graphs:
            assert sim.graph_steps >= 1, "no step ran as a whole-step graph"
    print(f"channel 256x128x128 ({'graphs' if graphs else 'eager'}), steps 1-4, worst relative error per field: " +
          ", ".join(f"{f} {e:.3e}" for f, e in worst.items()))


def test_channel_256x128x128_cell_flags(channel):
    """Device cell flags (inner bit, domain bit) equal the reference's inner
    and domain index lists on every multigrid level of the full-size scene."""
    xml, dump = channel
    g = A.Geometry(xml)
    cuda = A.load_cuda()
    with A.Simulation(xml) as sim:
        for level in range(g.levels + 1):
            dims = g.dims(level)
            n = dims[0] * dims[1] * dims[2]
            flags = np.zeros(n, np.uint8)
            A.cuda_check(cuda.artss_get_cell_flags(sim.context, level, flags.ctypes.data_as(C.POINTER(C.c_uint8)), n),
                         "flags")
            assert np.array_equal(np.flatnonzero(flags & 1), refdriver.ref_list(dump, "inner", level)), level
            assert np.array_equal(np.flatnonzero(flags & 2), refdriver.ref_list(dump, "domain", level)), level
