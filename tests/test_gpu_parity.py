"""Full-timestep parity of the B200 path with the reference serial build.

Each scene is an ARTSS XML written by artss_b200.scenes and run both by the
reference (oracle/_ref/artss_ref_driver: the unmodified ARTSS sources compiled
by oracle/Makefile) and by artss_b200.Simulation.  After every checked step
the fields u, v, w, p, T, nu_t (and rhs, S_T, buoyancy force) must agree to a
relative max-norm of 1e-10; in practice they agree bit for bit, because every
kernel evaluates the reference's expression with the same roundings and only
residual sums (which decide iteration counts, not values) are reduced in a
different order.
"""
import os

import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes
from tests import refdriver

pytestmark = pytest.mark.gpu

TOL = 1e-10
CHECK = ["u", "v", "w", "p", "T", "nu_t", "rhs", "S_T", "f_x", "f_y", "f_z"]


def _scenes():
    return {
        "box16_cgs": scenes.plume_box(n=16, steps=8, n_level=2),
        "box32_cgs": scenes.plume_box(n=32, steps=4, n_level=3),
        "channel_cube": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=4, n_level=3),
        "room_jacobi": scenes.room_with_door(n=32, steps=4, n_level=2),
        "room_cgs": scenes.room_with_door(n=32, steps=3, n_level=2, diffusion="ColoredGaussSeidel"),
        # the velocity-only solver compositions (src/solver/AdvectionSolver.cpp, ...)
        "advection": scenes.velocity_scene("AdvectionSolver", n=32, steps=4),
        "advection_diffusion": scenes.velocity_scene("AdvectionDiffusionSolver", n=32, steps=4),
        "diffusion_jacobi": scenes.velocity_scene("DiffusionSolver", n=32, steps=4),
        "diffusion_cgs": scenes.velocity_scene("DiffusionSolver", n=32, steps=4, diffusion="ColoredGaussSeidel"),
        "diffusion_turb": scenes.velocity_scene("DiffusionTurbSolver", n=32, steps=4),
        # NSTempTurbSolver without the turbulence model (src/solver/NSTempSolver.cpp)
        "nstemp_box": scenes.plume_box(n=32, steps=4, n_level=3, solver="NSTempSolver"),
        "nstemp_channel": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=3, n_level=3,
                                                   solver="NSTempSolver"),
        "nstemp_uniform_force": scenes.plume_box(n=32, steps=3, n_level=3, solver="NSTempSolver", force="Uniform",
                                                 buoyancy_dir="x,z", force_value=(0.1, 0.0, 0.3)),
        # the isothermal compositions (src/solver/NSSolver.cpp, NSTurbSolver.cpp) with
        # periodic boundaries and the Drift / McDermott / Vortex initial states
        "ns_cavity": scenes.ns_scene("cavity", n=32, steps=4),
        "ns_mcdermott": scenes.ns_scene("mcdermott", n=32, steps=4),
        "ns_channel": scenes.ns_scene("channel", n=32, steps=4),
        "nsturb_vortex": scenes.ns_scene("vortex", "NSTurbSolver", n=32, steps=4),
        "nsturb_cavity_cgs": scenes.ns_scene("cavity", "NSTurbSolver", n=32, steps=3, diffusion="ColoredGaussSeidel"),
        # ExplicitDiffuse (src/diffusion/ExplicitDiffuse.cpp) and the temperature's viscous
        # dissipation (ISource::dissipate, src/interfaces/ISource.cpp:63-123)
        "diffusion_explicit": scenes.velocity_scene("DiffusionSolver", n=32, steps=4, diffusion="Explicit"),
        "diffusion_turb_explicit": scenes.velocity_scene("DiffusionTurbSolver", n=32, steps=4, diffusion="Explicit"),
        "nstemp_dissipation": scenes.plume_box(n=32, steps=3, n_level=3, solver="NSTempSolver", dissipation=True),
        "nstempturb_explicit_dissipation": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=3, n_level=3,
                                                                    diffusion="Explicit", dissipation=True),
        # DynamicSmagorinsky (src/turbulence/DynamicSmagorinsky.cpp:172-427) in the turbulent timestep
        "nstempturb_dynamic_smagorinsky": scenes.channel_with_cube(nx=64, ny=32, nz=32, steps=3, n_level=3,
                                                                   turbulence="DynamicSmagorinsky"),
        "diffusion_turb_dynamic": scenes.velocity_scene("DiffusionTurbSolver", n=32, steps=3,
                                                        turbulence="DynamicSmagorinsky"),
        # PressureSolver (src/solver/PressureSolver.cpp:30-43) on the SinSinSin right-hand side
        "pressure_sinsinsin": scenes.pressure_scene(n=32, n_level=4, steps=2),
        # a computational domain inside the physical one (DomainData x1..z2), the LayersT
        # initial state (Functions::layers) with and without noise, buoyancy with
        # use_init_values (T_ambient never set: zero, as in the reference)
        "cd_layered_channel": scenes.layered_channel(steps=4),
        "cd_layered_channel_init_values": scenes.layered_channel(steps=3, use_init_values=True, noise=True),
        "cd_inset_box_obstacle": scenes.inset_box(steps=4),
        # AdvectionDiffusionSolver on ExpSinusSum (Functions::exp_sinus_sum), 2-D and 3-D
        "burgers_2d": scenes.burgers_scene(n=32, nz=1, steps=4),
        "burgers_3d": scenes.burgers_scene(n=32, nz=16, steps=4),
    }


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    if not refdriver.available():
        pytest.skip("reference oracle not built (oracle/Makefile)")
    base = tmp_path_factory.mktemp("parity")
    out = {}
    for name, sc in _scenes().items():
        xml = scenes.write(sc, str(base / f"{name}.xml"))
        dump = refdriver.run(xml, str(base / f"{name}_ref"), steps=sc.steps)
        out[name] = (xml, dump, sc)
    return out


@pytest.mark.parametrize("name", list(_scenes().keys()))
def test_timestep_parity(cases, name):
    xml, dump, sc = cases[name]
    with A.Simulation(xml) as sim:
        # set-up state (SolverController constructor)
        for f in CHECK:
            ref = refdriver.field(dump, 0, f)
            assert refdriver.rel_max_err(sim.field(f), ref) <= TOL, f"step 0 field {f}"
        worst = 0.0
        for step in range(1, sc.steps + 1):
            assert sim.run(1) == 1
            for f in CHECK:
                ref = refdriver.field(dump, step, f)
                err = refdriver.rel_max_err(sim.field(f), ref)
                worst = max(worst, err)
                assert err <= TOL, f"step {step} field {f}: relative max error {err:.3e}"
        print(f"{name}: worst relative error over {sc.steps} steps {worst:.3e}")


def test_cell_flags_match_reference_lists(cases):
    """The device cell flags are built from the host lists; they must mark
    exactly the reference's inner and domain lists on every level."""
    xml, dump, sc = cases["channel_cube"]
    ref_dir = refdriver.run(xml, dump + "_lists", steps=0, lists=True)
    g = A.Geometry(xml)
    cuda = A.load_cuda()
    with A.Simulation(xml) as sim:
        for level in range(g.levels + 1):
            dims = g.dims(level)
            n = dims[0] * dims[1] * dims[2]
            flags = np.zeros(n, np.uint8)
            A.cuda_check(cuda.artss_get_cell_flags(sim.context, level, flags.ctypes.data_as(
                __import__("ctypes").POINTER(__import__("ctypes").c_uint8)), n), "flags")
            inner = np.flatnonzero(flags & 1)
            domain = np.flatnonzero(flags & 2)
            assert np.array_equal(inner, refdriver.ref_list(ref_dir, "inner", level))
            assert np.array_equal(domain, refdriver.ref_list(ref_dir, "domain", level))
