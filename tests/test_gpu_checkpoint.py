"""Checkpoint and rollback (artss_sim_save / artss_sim_restore): the raw
stand-in for the reference's HDF5 data-assimilation checkpoints
(src/dataAssimilation/FieldIO.cpp:44-100).  A run that saves at step k,
continues, rolls back and repeats the same steps gives the fields of the
uninterrupted run bit for bit; a checkpoint of another grid is refused."""
import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes

pytestmark = pytest.mark.gpu
FIELDS = ["u", "v", "w", "p", "T", "nu_t", "rhs", "S_T"]


@pytest.mark.parametrize("graphs", [False, True], ids=["eager", "graphs"])
def test_rollback_repeats_the_run(tmp_path, graphs):
    sc = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=12, n_level=3)
    xml = scenes.write(sc, str(tmp_path / "ch.xml"))
    ck = str(tmp_path / "step4.ckp")
    with A.Simulation(xml) as sim:
        sim.set_graphs(graphs)
        assert sim.run(3) == 3
        sim.save(ck)
        saved_step, saved_t = sim.step_index, sim.time
        assert sim.run(4) == 4
        first = {f: sim.field(f) for f in FIELDS}
        sim.restore(ck)
        assert (sim.step_index, sim.time) == (saved_step, saved_t)
        assert sim.run(4) == 4
        for f in FIELDS:
            assert np.array_equal(sim.field(f), first[f]), f


def test_restore_into_a_fresh_simulation(tmp_path):
    sc = scenes.plume_box(n=32, steps=10, n_level=3)
    xml = scenes.write(sc, str(tmp_path / "box.xml"))
    ck = str(tmp_path / "box.ckp")
    with A.Simulation(xml) as sim:
        sim.run(4)
        sim.save(ck)
        sim.run(3)
        ref = {f: sim.field(f) for f in FIELDS}
    with A.Simulation(xml) as sim:
        sim.restore(ck)
        assert sim.run(3) == 3
        for f in FIELDS:
            assert np.array_equal(sim.field(f), ref[f]), f


def test_restore_rejects_another_grid(tmp_path):
    a = scenes.write(scenes.plume_box(n=16, steps=4, n_level=2), str(tmp_path / "a.xml"))
    b = scenes.write(scenes.plume_box(n=32, steps=4, n_level=2), str(tmp_path / "b.xml"))
    ck = str(tmp_path / "a.ckp")
    with A.Simulation(a) as sim:
        sim.run(1)
        sim.save(ck)
    with A.Simulation(b) as sim:
        with pytest.raises(A.ArtssError, match="grid"):
            sim.restore(ck)
