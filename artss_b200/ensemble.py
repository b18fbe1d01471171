"""Ensembles of independent scenes (data assimilation, parameter studies).

No counterpart in the reference, which runs one scene per process.  Scenes
are independent, so they shard across GPUs with no data-path collective: a
greedy longest-processing-time partition by cell count assigns scenes to
ranks, and on one GPU every scene runs in its own context (own CUDA stream)
driven by its own host thread, so the kernels of different scenes overlap on
the device while each scene's host code waits on its own loop controls.
"""
from __future__ import annotations

import heapq
from concurrent.futures import ThreadPoolExecutor
from typing import List, Sequence


def partition(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment of items to `parts` bins:
    items in decreasing cost, each to the currently lightest bin (ties: lower
    bin index).  Returns the item indices of every bin, in ascending order."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    heap = [(0.0, b) for b in range(parts)]
    heapq.heapify(heap)
    bins: List[List[int]] = [[] for _ in range(parts)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, b = heapq.heappop(heap)
        bins[b].append(i)
        heapq.heappush(heap, (load + float(costs[i]), b))
    return [sorted(b) for b in bins]


class Ensemble:
    """Independent scenes on one GPU, stepped concurrently.  With graphs=True
    every scene's step is one CUDA graph launch from the third step on.  The
    scenes' streams overlap best with CUDA_DEVICE_MAX_CONNECTIONS=32 in the
    environment before the process creates its CUDA context."""

    def __init__(self, xml_paths: Sequence[str], device: int = 0, graphs: bool = False):
        from artss_b200 import Simulation
        self.sims = [Simulation(x, device=device) for x in xml_paths]
        if graphs:
            # from the third step on, every scene's step is one graph launch
            for s in self.sims:
                s.set_graphs(True)

    @property
    def inner_cells(self) -> int:
        return sum(s.inner_cells for s in self.sims)

    def streams(self):
        from artss_b200 import load_cuda
        lib = load_cuda()
        return [lib.artss_ctx_stream(s.context) for s in self.sims]

    def run(self, steps: int) -> List[int]:
        """Advances every scene by `steps` timesteps, one host thread per scene;
        returns the steps each scene did."""
        if not self.sims:
            return []
        with ThreadPoolExecutor(max_workers=len(self.sims)) as ex:
            return list(ex.map(lambda s: s.run(steps), self.sims))

    def close(self):
        for s in self.sims:
            s.close()
        self.sims = []
