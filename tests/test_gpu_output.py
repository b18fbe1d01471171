"""Output side of the time loop against the reference build's own routines:
the device CFL max-reduction against Analysis::calc_CFL
(src/analysis/Analysis.cpp:322-351), and the files of Analysis::write_file
(:378-387) and VTKWriter::write_numerical (src/visualisation/VTKWriter.cpp:
60-106) byte for byte.  The writers take a snapshot read-back, so a write
queued at step k holds step k's values although the run goes on before the
file is written."""
import json
import os
import subprocess

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import refdriver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_outputs(tmp_path_factory):
    if not refdriver.available():
        pytest.skip("reference oracle not built (oracle/Makefile)")
    base = tmp_path_factory.mktemp("outputs")
    sc = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=8, n_level=3)
    xml = scenes.write(sc, str(base / "ch.xml"))
    r = subprocess.run([refdriver.DRIVER, xml, "--steps", "3", "--vtk", str(base / "ref3"), "--dat",
                        f"T:{base / 'ref3_T'}", "--cfl"], check=True, capture_output=True, text=True, timeout=600)
    cfl = json.loads(r.stdout.strip().splitlines()[-1])["cfl"]
    return xml, base, cfl


def _bytes(path):
    with open(path, "rb") as f:
        return f.read()


def test_cfl_matches_reference(ref_outputs):
    xml, base, ref_cfl = ref_outputs
    with A.Simulation(xml) as sim:
        sim.run(3)
        got = sim.cfl()
        u, v, w = sim.field("u"), sim.field("v"), sim.field("w")
        g = A.Geometry(xml)
        inner = g.list("inner", 0)
        d = g.grid_desc()
        dt = 0.002  # the channel scene's time step
        mine = dt * float(np.max(np.abs(u[inner]) / d.dx[0] + np.abs(v[inner]) / d.dy[0] + np.abs(w[inner]) / d.dz[0]))
    assert got == ref_cfl, (got, ref_cfl)
    assert got == mine


def test_writers_match_reference_after_more_steps(ref_outputs):
    """write_vtk / write_dat queued after step 3; two more steps run before the
    worker writes the files; the files equal the reference's step-3 files."""
    xml, base, _ = ref_outputs
    ours_vtk, ours_dat = str(base / "ours3"), str(base / "ours3_T.dat")
    with A.Simulation(xml) as sim:
        sim.run(3)
        sim.write_vtk(ours_vtk)
        sim.write_dat("T", ours_dat)
        sim.run(2)
        sim.output_wait()
    assert _bytes(ours_vtk + ".vtk") == _bytes(str(base / "ref3.vtk"))
    assert _bytes(ours_dat) == _bytes(str(base / "ref3_T.dat"))


def test_many_queued_writes(tmp_path):
    """More writes than read-back slots in flight: each call waits for the
    slot two before it; every file holds its own step's values."""
    sc = scenes.plume_box(n=16, steps=10, n_level=2)
    xml = scenes.write(sc, str(tmp_path / "box.xml"))
    expect = {}
    with A.Simulation(xml) as sim:
        for k in range(6):
            sim.run(1)
            expect[k] = sim.field("T")
            sim.write_dat("T", str(tmp_path / f"T{k}.dat"))
        sim.output_wait()
    for k, T in expect.items():
        vals = np.loadtxt(str(tmp_path / f"T{k}.dat"))
        assert vals.shape == T.shape
        assert np.allclose(vals, T, rtol=1e-5, atol=0), k
