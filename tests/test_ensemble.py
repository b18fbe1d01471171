"""Ensembles of independent scenes: the scene-to-rank partition (host logic,
also across two gloo ranks on the CPU) and, on the GPU, concurrent stepping
that must give every scene exactly the fields it gets when run alone."""
import os
import socket

import numpy as np
import pytest

from artss_b200.ensemble import partition


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(32, 129, size=(64, 3)).prod(axis=1).astype(float)
    for parts in (1, 2, 3, 8):
        bins = partition(costs, parts)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(len(costs)))
        loads = [costs[b].sum() for b in bins]
        # the greedy LPT bound: max load <= (4/3 - 1/(3 parts)) * optimum <= that times the mean
        assert max(loads) <= (4 / 3) * max(costs.sum() / parts, costs.max()) + 1e-9


def test_partition_empty_and_errors():
    assert partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition(costs, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    # every rank reports the cells it would process; rank 0 checks the split
    load = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
    dist.all_reduce(load)
    if rank == 0:
        q.put((gathered, float(load.item())))
    dist.destroy_process_group()


def test_partition_two_gloo_ranks():
    import multiprocessing as mp
    costs = [float(c) for c in np.random.default_rng(1).integers(1000, 100000, size=17)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(i for g in gathered for i in g) == list(range(len(costs)))
    assert total == pytest.approx(sum(costs))


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [False, True])
def test_ensemble_concurrent_matches_alone(tmp_path, graphs):
    """Scenes stepped concurrently (optionally as whole-step graphs from the
    third step on) give exactly the fields of each scene run alone, step by step."""
    import artss_b200 as A
    from artss_b200 import scenes
    from artss_b200.ensemble import Ensemble
    steps = 6 if graphs else 3
    scs = scenes.plume_ensemble(3, seed=5, steps=steps, sizes=(32, 48))
    xmls = [scenes.write(sc, str(tmp_path / f"e{i}.xml")) for i, sc in enumerate(scs)]
    ens = Ensemble(xmls, graphs=graphs)
    try:
        assert ens.run(steps) == [steps] * 3
        if graphs:
            assert all(s.graph_steps == steps - 2 for s in ens.sims)
        together = [{f: s.field(f) for f in ("u", "p", "T")} for s in ens.sims]
    finally:
        ens.close()
    for x, ref in zip(xmls, together):
        with A.Simulation(x) as sim:
            sim.run(steps)
            for f in ("u", "p", "T"):
                assert np.array_equal(sim.field(f), ref[f]), f
