"""One timestep with its host transfers (artss_sim_step_io): inputs uploaded
during the step and outputs read back beside it must give exactly what
setting the fields (and the copies u0, u_tmp, ..., T0, T_tmp of the state),
running the step and reading them back gives."""
import numpy as np
import pytest

import artss_b200 as A
from artss_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "T")


@pytest.mark.parametrize("solver", ["NSTempTurbSolver", "NSTempSolver"])
def test_step_io_matches_set_run_get(tmp_path, solver):
    import torch
    sc = scenes.plume_box(n=32, steps=8, n_level=3, solver=solver)
    xml = scenes.write(sc, str(tmp_path / "s.xml"))
    with A.Simulation(xml) as a, A.Simulation(xml) as b:
        assert a.run(2) == 2 and b.run(2) == 2
        rng = np.random.default_rng(7)
        for step in range(3):
            # inputs that differ from the device state, so that every upload matters
            ins = {f: torch.from_numpy(a.field(f) * (1 + 1e-3 * rng.standard_normal(a.size))).pin_memory()
                   for f in FIELDS}
            outs = {f: torch.empty(a.size, dtype=torch.float64).pin_memory() for f in FIELDS}
            a.step_io({f: t.data_ptr() for f, t in ins.items()}, {f: t.data_ptr() for f, t in outs.items()})
            for f in FIELDS:
                b.set_field(f, ins[f].numpy())
            # the state the step advances: the copies follow the uploaded u, v, w, T
            for f in ("u", "v", "w", "T"):
                b.set_field(f + "0", ins[f].numpy())
                b.set_field(f + "_tmp", ins[f].numpy())
            assert b.run(1) == 1
            for f in FIELDS:
                ref = b.field(f)
                assert np.array_equal(outs[f].numpy(), ref), (step, f)
                assert np.array_equal(a.field(f), ref), (step, f)


@pytest.mark.parametrize("solver", ["NSTempTurbSolver", "NSTempSolver"])
def test_step_io_async_matches_step_io(tmp_path, solver):
    """Pipelined steps (artss_sim_step_io_async): four calls in flight through
    both staging sets give, step for step, what the synchronous call gives."""
    import torch
    sc = scenes.plume_box(n=32, steps=12, n_level=3, solver=solver)
    xml = scenes.write(sc, str(tmp_path / "s.xml"))
    with A.Simulation(xml) as a, A.Simulation(xml) as b:
        assert a.run(2) == 2 and b.run(2) == 2
        rng = np.random.default_rng(11)
        n_steps = 5
        ins = [{f: torch.from_numpy(a.field(f) * (1 + 1e-3 * rng.standard_normal(a.size))).pin_memory()
                for f in FIELDS} for _ in range(n_steps)]
        outs_a = [{f: torch.empty(a.size, dtype=torch.float64).pin_memory() for f in FIELDS} for _ in range(n_steps)]
        outs_b = [{f: torch.empty(a.size, dtype=torch.float64).pin_memory() for f in FIELDS} for _ in range(n_steps)]
        for k in range(n_steps):
            a.step_io_async({f: t.data_ptr() for f, t in ins[k].items()},
                            {f: t.data_ptr() for f, t in outs_a[k].items()})
        a.io_sync()
        for k in range(n_steps):
            b.step_io({f: t.data_ptr() for f, t in ins[k].items()}, {f: t.data_ptr() for f, t in outs_b[k].items()})
        for k in range(n_steps):
            for f in FIELDS:
                assert np.array_equal(outs_a[k][f].numpy(), outs_b[k][f].numpy()), (k, f)
        for f in FIELDS:
            assert np.array_equal(a.field(f), b.field(f)), f
        assert a.step_index == b.step_index
