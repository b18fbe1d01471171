"""Whole-step CUDA graphs: from the third step on a step is one graph launch
whose diffusion and pressure loops are conditional WHILE nodes decided by the
device loop state.  Every field must equal the step-by-step run bit for bit,
for every solver and loop kind the graphs capture."""
import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ["u", "v", "w", "p", "T", "nu_t", "rhs", "S_T", "f_x", "f_y", "f_z"]


def _scenes():
    return {
        "box_cgs": scenes.plume_box(n=32, steps=9, n_level=3),
        "channel_cube": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=8, n_level=3),
        "box_mixed_pressure": scenes.plume_box(n=32, steps=9, n_level=3, pressure="VCycleMGMixed", max_cycle=20),
        "room_jacobi": scenes.room_with_door(n=32, steps=8, n_level=2),
        "ns_cavity": scenes.ns_scene("cavity", n=32, steps=8),
    }


@pytest.mark.parametrize("name", list(_scenes().keys()))
def test_graph_steps_equal_eager_steps(tmp_path, name):
    sc = _scenes()[name]
    xml = scenes.write(sc, str(tmp_path / f"{name}.xml"))
    with A.Simulation(xml) as eager, A.Simulation(xml) as graph:
        graph.set_graphs(True)
        for chunk in (2, 3, sc.steps - 5):
            assert eager.run(chunk) == chunk
            assert graph.run(chunk) == chunk
            for f in FIELDS:
                a, b = eager.field(f), graph.field(f)
                assert np.array_equal(a, b), (name, f, eager.step_index)
        # steps 3.. ran as graph launches
        assert graph.graph_steps == sc.steps - 2


@pytest.mark.parametrize("name", ["box_cgs", "channel_cube"])
def test_programmatic_launch_changes_nothing(tmp_path, name):
    """Kernels launched to overlap their predecessor's tail (artss_ctx_pdl 2,
    the default, eager and inside graphs) give the fields that plain launches
    (mode 0) give."""
    sc = _scenes()[name]
    xml = scenes.write(sc, str(tmp_path / f"{name}.xml"))
    with A.Simulation(xml) as plain, A.Simulation(xml) as pdl, A.Simulation(xml) as pdl_graph:
        lib = plain._lib
        assert lib.artss_ctx_pdl(plain.context, 0) == 0
        pdl_graph.set_graphs(True)
        for s in (plain, pdl, pdl_graph):
            assert s.run(sc.steps - 1) == sc.steps - 1
        for f in FIELDS:
            ref = plain.field(f)
            assert np.array_equal(pdl.field(f), ref), (name, f)
            assert np.array_equal(pdl_graph.field(f), ref), (name, f)
        assert pdl_graph.graph_steps == sc.steps - 3
