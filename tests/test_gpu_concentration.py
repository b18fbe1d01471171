"""NSTempTurbConSolver / NSTempConSolver (src/solver/NSTempTurbConSolver.cpp,
NSTempConSolver.cpp): the temperature solvers plus a passive concentration
stage (advection with the new velocity, diffusion with gamma or gamma + nu_t /
Sc_T, the source, couples).

The reference cannot run either solver: both constructors store the
concentration's advection in adv_temp a second time and never set adv_con
(NSTempTurbConSolver.cpp:29, NSTempConSolver.cpp:30), so do_step calls through
an unset pointer.  Parity is anchored instead on
* u, v, w, p, T: the concentration is passive, so the Con solver's velocity,
  pressure and temperature equal the reference build's NSTempTurbSolver /
  NSTempSolver on the same scene without the concentration block, bit for bit;
* C: with the concentration set up exactly like the temperature (same initial
  value, boundary conditions, source, gamma = kappa, Sc_T = Pr_T), C equals T
  bit for bit after every step, since it runs the same kernels in the same
  order on the same inputs."""
import dataclasses

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import refdriver

pytestmark = pytest.mark.gpu

FIELDS = ["u", "v", "w", "p", "T"]


def _zero_temperature_channel(**kw):
    """The 64x32x32 channel with the cube, T = 0 initially, at the inflow and
    as the ambient value (so that C, which starts at zero, and T coincide)."""
    sc = scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=3, n_level=3, T0=0.0, t_ambient=0.0, **kw)
    bcs = [(f, p, t, 0.0 if f == "T" else v) for f, p, t, v in sc.boundaries]
    return dataclasses.replace(sc, boundaries=bcs)


def _scenes():
    return {
        "turbulent": _zero_temperature_channel(),
        "laminar": _zero_temperature_channel(solver="NSTempSolver"),
    }


@pytest.mark.parametrize("name", list(_scenes().keys()))
def test_concentration_equals_temperature_configured_alike(tmp_path, name):
    # no initial noise on T: C starts at exactly zero
    sc = dataclasses.replace(_scenes()[name], concentration=True, noise=False)
    xml = scenes.write(sc, str(tmp_path / f"con_{name}.xml"))
    assert ("NSTempTurbConSolver" if name == "turbulent" else "NSTempConSolver") in open(xml).read()
    with A.Simulation(xml) as sim:
        assert np.array_equal(sim.field("C"), sim.field("T"))
        for step in range(1, sc.steps + 1):
            assert sim.run(1) == 1
            C, T = sim.field("C"), sim.field("T")
            assert np.array_equal(C, T), f"step {step}: C differs from T"
        # the source ramps in with tanh(t / tau): zero in the first step only
        assert np.abs(T).max() > 0, "the source did not act"


@pytest.mark.parametrize("name", list(_scenes().keys()))
def test_concentration_solver_velocity_and_temperature_match_reference(tmp_path, name):
    if not refdriver.available():
        pytest.skip("reference oracle not built (oracle/Makefile)")
    plain = _scenes()[name]
    ref_xml = scenes.write(plain, str(tmp_path / f"plain_{name}.xml"))
    dump = refdriver.run(ref_xml, str(tmp_path / "ref"), steps=plain.steps, every=1, fields=FIELDS)
    xml = scenes.write(dataclasses.replace(plain, concentration=True), str(tmp_path / f"con_{name}.xml"))
    with A.Simulation(xml) as sim:
        for step in range(0, plain.steps + 1):
            if step:
                assert sim.run(1) == 1
            for f in FIELDS:
                err = refdriver.rel_max_err(sim.field(f), refdriver.field(dump, step, f))
                assert err == 0.0, f"step {step} field {f}: relative max error {err:.3e}"
