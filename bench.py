"""Benchmark of the ARTSS fractional-step timestep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload channel|box]

A step is one NSTempTurbSolver timestep (SolverController::solver_do_step +
update_sources + update_data, ARTSS src/TimeIntegration.cpp:86-145) of the
workload scene.  Default workload: the plain-FP64 channel, 256x128x128 cells,
one 0.4 m cube, Dirichlet inflow, 100 kW Gaussian source, dt = 0.002 s
(artss_b200.scenes.channel_with_cube); the metric is cell-updates/s =
inner cells x steps / time.  Warm-up steps include step 1, whose pressure
solve iterates to tolerance.

N > 1 (torchrun): the single scene does not shard, every rank runs its own
replica on its own GPU and `value` is the sum over ranks (weak scaling).
`--impl reference` times the reference serial build (oracle/_ref) on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
STATE_FIELDS = ["u", "v", "w", "p", "T"]
# stages of NSTempTurbSolver::do_step + the time loop's update (ARTSS_STAGE_* of artss_cuda.h)
STAGES = ["advection", "diffusion", "momentum_source", "pressure", "temperature", "update"]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["channel", "box", "poisson", "ensemble", "learned"], default="channel",
                    help="poisson: ms per pressure solve to a 1e-8 relative residual, plain FP64 VCycleMG "
                         "against the mixed-precision solve, on the 256^3 Neumann problem with box obstacles")
    ap.add_argument("--poisson-n", type=int, default=256)
    ap.add_argument("--poisson-levels", type=int, default=5)
    ap.add_argument("--channel-nx", type=int, default=256,
                    help="channel workload size nx x nx/2 x nx/2 (256: the benchmarked scene; smaller sizes for "
                         "profiler captures)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=3, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload(name: str, steps: int, nx: int = 256):
    from artss_b200 import scenes
    if name == "channel":
        return (f"channel_{nx}x{nx // 2}x{nx // 2}_cube_fp64",
                scenes.channel_with_cube(nx=nx, ny=nx // 2, nz=nx // 2, steps=steps))
    return "box_64cubed_plume_fp64", scenes.plume_box(n=64, steps=steps, n_level=4)


def step_config(name: str, sc, inner: int, world: int) -> dict:
    """The `config` object of a timestep line; both arms print the same one."""
    return {"workload": name, "cells": f"{sc.nx}x{sc.ny}x{sc.nz}", "inner_cells": inner,
            "obstacles": len(sc.obstacles), "dt": sc.dt, "mg_levels": sc.n_level,
            "diffusion": sc.diffusion, "parallelism": "replicas" if world > 1 else "single",
            "l2": "no flush: the ~25 resident FP64 arrays (~870 MB) exceed the 126 MB L2"}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                cols = [c.strip() for c in line.split(",")]
                if len(cols) < 9:
                    continue
                try:
                    sm.append(float(cols[1]))
                    mx = float(cols[2])
                except ValueError:
                    continue
                for n, c in zip(names, cols[5:9]):
                    if c.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class Dist:
    """torch.distributed plumbing for N > 1 (one rank per GPU)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            self.pg.barrier(device_ids=[self.local])
            torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# Algorithmic bytes of one launch, per inner cell of level 0 (n) or per array
# cell (N) -- FP64, each array element read or written once; neighbour
# re-reads are not counted.
def launch_bytes(family: str, n: int, N: int, launches: int) -> float:
    if family == "advect":       # per step: fused u,v,w (read u0,v0,w0; write u,v,w: 48 B) + T (read u,v,w,T0; write T: 40 B)
        return launches / 2 * (48 + 40) * n
    if family == "cgs_sweep":    # one red+black iteration: read x, b, EV (turbulent), write x: 32 B
        return launches * 32.0 * n
    if family == "smagorinsky":  # read u, v, w; write nu_t
        return launches * 32.0 * n
    if family == "couple":       # per step 4 vector couples (read 3, write 6 arrays) + 4 scalar (read 1, write 2)
        return launches / 2 * (72 + 24) * N
    if family == "projection":   # read u*, v*, w*, p; write u, v, w
        return launches * 56.0 * n
    return 0.0


# DRAM bytes (read + write) per launch from one ncu capture of the kernel on
# the 256x128x128 channel, per inner cell: profiles/k_cgs_sweep_tma_channel256x128x128.md
NCU_TRAFFIC_PER_CELL = {"cgs_sweep": (118.077440e6 + 13.617152e6) / 4190208}

MODELED = ("advect", "cgs_sweep", "smagorinsky", "couple", "projection")


def run_b200(args, dist):
    import numpy as np
    import torch

    import artss_b200 as A
    from artss_b200 import scenes

    torch.cuda.set_device(dist.local)
    total_steps = args.warmup + 2 + 3 * args.steps + 2 * args.e2e_steps + 3 + 2
    name, sc = workload(args.workload, total_steps, args.channel_nx)
    tmp = tempfile.mkdtemp(prefix="artss_bench_")
    xml = scenes.write(sc, os.path.join(tmp, f"{name}_r{dist.rank}.xml"))
    sim = A.Simulation(xml, device=dist.local)
    cuda = A.load_cuda()
    ctx = sim.context
    inner = sim.inner_cells
    size = sim.size
    stream = torch.cuda.ExternalStream(cuda.artss_ctx_stream(ctx), device=torch.device("cuda", dist.local))

    sim.run(args.warmup)

    # family shares over two untimed steps, then events on the dominant modeled family only
    nf = 20
    cuda.artss_ctx_profile(ctx, (1 << nf) - 1)
    cuda.artss_ctx_profile_reset(ctx)
    sim.run(2)
    L = (C.c_int64 * nf)()
    M = (C.c_double * nf)()
    A.cuda_check(cuda.artss_ctx_profile_read(ctx, L, M, nf), "profile")
    fam_names = [cuda.artss_kernel_family_name(f).decode() for f in range(nf)]
    share_ms = {fam_names[f]: M[f] for f in range(nf) if L[f]}
    dom = max((f for f in range(nf) if fam_names[f] in MODELED and L[f]), key=lambda f: M[f])
    # the timed steps run without per-launch events (they would split the
    # programmatic launch overlap); the dominant kernel is timed after them
    cuda.artss_ctx_profile(ctx, 0)

    sampler = ClockSampler(dist.local)
    sampler.start()
    launches0 = sim.kernel_launches()
    dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # NVTX range: a profiler can restrict itself to the timed steps (ncu --nvtx-include "timed_steps/")
    torch.cuda.nvtx.range_push("timed_steps")
    done = sim.run(args.steps)
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    assert done == args.steps, "scene ended early"
    ms = e0.elapsed_time(e1)
    gpu_launches = sim.kernel_launches() - launches0
    # the same number of steps again with CUDA events around every launch of
    # the dominant kernel on the simulation's stream: its average duration
    cuda.artss_ctx_profile(ctx, 1 << dom)
    cuda.artss_ctx_profile_reset(ctx)
    assert sim.run(args.steps) == args.steps, "scene ended early"
    torch.cuda.synchronize()
    A.cuda_check(cuda.artss_ctx_profile_read(ctx, L, M, nf), "profile")
    dom_launches, dom_ms = int(L[dom]), float(M[dom])
    cuda.artss_ctx_profile(ctx, 0)
    # the same number of steps once more with one event per stage boundary
    # (artss_ctx_stage_mark, six per step): device ms per stage
    A.cuda_check(cuda.artss_ctx_stage_timing(ctx, 1), "stage timing")
    assert sim.run(args.steps) == args.steps, "scene ended early"
    S = (C.c_double * 6)()
    A.cuda_check(cuda.artss_ctx_stage_read(ctx, S, 6), "stage read")
    A.cuda_check(cuda.artss_ctx_stage_timing(ctx, 0), "stage timing")
    stage_ms = {n: round(S[i] / args.steps, 4) for i, n in enumerate(STAGES)}

    # end to end, pipelined (the headline): every step uploads its state from
    # page-locked host memory, runs one timestep and reads the state back
    # through Simulation.step_io_async; step k+1's upload and step k's
    # read-back run on the two copy engines beside the steps.  Call k reads and
    # overwrites host set k % 3, so the state read back feeds the step three
    # later (the k-th call returns once call k-2 is complete).
    # Each step is one whole-step graph launch (Simulation.set_graphs), so the
    # host enqueues the next step's upload while the device runs this one;
    # three untimed calls capture the graph first.
    sets = [{f: torch.from_numpy(sim.field(f)).pin_memory() for f in STATE_FIELDS} for _ in range(3)]
    sim.set_graphs(True)
    for s_ in range(3):
        io = {f: sets[s_ % 3][f].data_ptr() for f in STATE_FIELDS}
        sim.step_io_async(io, io)
    sim.io_sync()
    graph_steps0 = sim.graph_steps
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for s_ in range(args.e2e_steps):
        io = {f: sets[s_ % 3][f].data_ptr() for f in STATE_FIELDS}
        sim.step_io_async(io, io)
    sim.io_sync()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_graph_steps = sim.graph_steps - graph_steps0
    sim.set_graphs(False)
    if not all(np.isfinite(st["T"].numpy()).all() for st in sets):
        raise RuntimeError("non-finite temperature after the end-to-end steps")

    # end to end, serial: each step's input is the previous step's read-back
    # (Simulation.step_io: p and T arrive while the velocity is computed, u,
    # v, w, p leave while T is; complete on return)
    pinned = [{f: torch.from_numpy(sim.field(f)).pin_memory() for f in STATE_FIELDS},
              {f: torch.empty(size, dtype=torch.float64).pin_memory() for f in STATE_FIELDS}]
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for s_ in range(args.e2e_steps):
        src, dst = pinned[s_ & 1], pinned[(s_ + 1) & 1]
        sim.step_io({f: src[f].data_ptr() for f in STATE_FIELDS}, {f: dst[f].data_ptr() for f in STATE_FIELDS})
    e1.record(stream)
    e1.synchronize()
    e2e_serial_ms = e0.elapsed_time(e1)
    if not np.isfinite(pinned[args.e2e_steps & 1]["T"].numpy()).all():
        raise RuntimeError("non-finite temperature after the end-to-end steps")

    ms_max = dist.max(ms)
    e2e_ms_max = dist.max(e2e_ms)
    e2e_serial_ms_max = dist.max(e2e_serial_ms)
    cells_all = dist.sum(float(inner) * args.steps)
    e2e_cells_all = dist.sum(float(inner) * args.e2e_steps)
    hbm, peak_kind = peaks()
    fam = fam_names[dom]
    achieved = launch_bytes(fam, inner, size, dom_launches) / (dom_ms * 1e-3) / 1e9 if dom_ms > 0 else 0.0
    out = {
        "metric": "cell-updates/s per timestep",
        "value": cells_all / (ms_max * 1e-3),
        "unit": "cell-updates/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": step_config(name, sc, inner, dist.world),
        "clocks": clocks,
        "e2e": {"value": e2e_cells_all / (e2e_ms_max * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": len(STATE_FIELDS) * size * 8,
                "d2h_bytes_per_step": len(STATE_FIELDS) * size * 8,
                "what": "per step through Simulation.step_io_async (artss_sim_step_io_async): u,v,w,p,T uploaded "
                        "from page-locked host memory as the state the step advances, one timestep, u,v,w,p,T read "
                        "back; uploads and read-backs on the two copy engines beside the steps (each step one "
                        "whole-step graph launch), the state read back feeding the step three later; timed to the "
                        "last read-back",
                "graph_steps": int(e2e_graph_steps),
                "serial": {"value": e2e_cells_all / (e2e_serial_ms_max * 1e-3), "unit": "cell-updates/s",
                           "what": "Simulation.step_io (artss_sim_step_io), complete on return, each step's input "
                                   "the previous step's read-back (p and T arrive while the velocity is computed, "
                                   "u,v,w,p leave while T is)"}},
        "gpu_launches": int(gpu_launches),
        "roofline": {"bound": "hbm", "kernel": fam, "achieved": achieved, "peak": hbm,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": (NCU_TRAFFIC_PER_CELL[fam] * inner if fam in NCU_TRAFFIC_PER_CELL else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, per inner "
                                       "cell, scaled to this workload's cells",
                     "launches": dom_launches, "avg_launch_us": 1e3 * dom_ms / max(dom_launches, 1),
                     "timing": "CUDA events around each launch on the simulation's stream, over a second run of "
                               "the timed steps (the first runs without them)"},
        "stage_ms_per_step": stage_ms,
        "stage_timing": "device ms per stage and step: one CUDA event per stage boundary on the simulation's stream "
                        "over a third run of the timed steps",
        "kernel_family_ms_two_steps": {k: round(v, 4) for k, v in sorted(share_ms.items(), key=lambda kv: -kv[1])},
        "kernel_family_note": "CUDA events around every launch over two untimed steps; the events serialise the "
                              "programmatic launch overlap, so these sums exceed the step time (shares only)",
    }
    sim.close()
    return out, xml, inner


def run_poisson(args, dist):
    """ms per pressure solve to ||b - A p|| <= 1e-8 ||b|| from p = 0: the plain
    FP64 VCycleMG (reference V-cycle structure: 5 levels, V(2,2) Jacobi
    w = 2/3, 100-sweep Jacobi coarse solve; the reference's smoothing keeps
    the first of each pair of relaxations) against the mixed-precision solve
    (FP32 V(2,2) cycles of the same depth with Jacobi weight 6/7, FP64 defect
    correction, red-black SOR coarse solve to 1e-2 relative).  `steps` solves of each are timed with CUDA events on the
    context stream, after `warmup` untimed ones."""
    import numpy as np
    import torch

    import artss_b200 as A
    from artss_b200 import scenes

    torch.cuda.set_device(dist.local)
    n = args.poisson_n
    nl = args.poisson_levels
    sc = scenes.poisson_boxes(n=n, seed=args.seed, n_level=nl)
    xml = scenes.write(sc, os.path.join(tempfile.mkdtemp(prefix="artss_poisson_"), "poisson.xml"))
    geom = A.Geometry(xml)
    ctx = A.Context(geom, device=dist.local)
    cuda = ctx.lib
    stream = torch.cuda.ExternalStream(cuda.artss_ctx_stream(ctx.h), device=torch.device("cuda", dist.local))
    inner = geom.list("inner", 0)
    b_raw = scenes.poisson_rhs(inner, ctx.size(), 1000 + args.seed)
    db, b = A.consistent_rhs(ctx, b_raw, nl)
    dp = ctx.field()
    mg = C.c_void_p()
    mcfg = A.MgCfg(nl, 2, 100, 2, 1e-8, 0, 0, 100, 1e-8, 0.6666666667)
    A.cuda_check(cuda.artss_mg_create(ctx.h, C.byref(mcfg), C.byref(mg)), "mg")
    mx = C.c_void_p()
    # Jacobi weight 6/7 (the smoothing-optimal weight of the 7-point operator);
    # coarse red-black SOR to 1e-2 relative, at most 20 sweeps
    xcfg = A.MixedCfg(nl, 2, 1, A.MIXED_REMOVE_MEAN, 6.0 / 7.0, 0.0, 1e-2, 20, 1e-8, 200)
    A.cuda_check(cuda.artss_mixed_create(ctx.h, C.byref(xcfg), C.byref(mx)), "mixed")
    # red-black Gauss-Seidel smoothing (w = 1), one or two sweeps each side
    mx_rb = {}
    for nr in (1, 2):
        h = C.c_void_p()
        rcfg = A.MixedCfg(nl, nr, 1, A.MIXED_REMOVE_MEAN | A.MIXED_RBGS, 1.0, 0.0, 1e-2, 20, 1e-8, 200)
        A.cuda_check(cuda.artss_mixed_create(ctx.h, C.byref(rcfg), C.byref(h)), "mixed rbgs")
        mx_rb[nr] = h

    def plain(st):
        return cuda.artss_mg_solve_rel(mg, dp, db, 1e-8, 2000, C.byref(st))

    def mixed(st):
        return cuda.artss_mixed_solve(mx, dp, db, C.byref(st))

    def rbgs(nr):
        return lambda st: cuda.artss_mixed_solve(mx_rb[nr], dp, db, C.byref(st))

    res = {}
    for name, fn in (("plain_fp64", plain), ("mixed", mixed), ("mixed_rbgs_v11", rbgs(1)),
                     ("mixed_rbgs_v22", rbgs(2))):
        st = A.SolveStats()
        for _ in range(args.warmup):
            A.cuda_check(cuda.artss_fill(ctx.h, dp, 0, 0.0), "fill")
            A.cuda_check(fn(st), name)
        times = []
        for _ in range(args.steps):
            A.cuda_check(cuda.artss_fill(ctx.h, dp, 0, 0.0), "fill")
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            A.cuda_check(fn(st), name)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        # one more solve with per-family event timing (not part of the timed numbers)
        nf = 20
        cuda.artss_ctx_profile(ctx.h, (1 << nf) - 1)
        cuda.artss_ctx_profile_reset(ctx.h)
        A.cuda_check(cuda.artss_fill(ctx.h, dp, 0, 0.0), "fill")
        A.cuda_check(fn(st), name)
        Lc = (C.c_int64 * nf)()
        Mc = (C.c_double * nf)()
        A.cuda_check(cuda.artss_ctx_profile_read(ctx.h, Lc, Mc, nf), "profile")
        cuda.artss_ctx_profile(ctx.h, 0)
        fam = {cuda.artss_kernel_family_name(f).decode(): (int(Lc[f]), round(Mc[f], 3)) for f in range(nf) if Lc[f]}
        res[name] = {"ms_per_solve": float(np.median(times)), "ms_all": [round(t, 3) for t in times],
                     "cycles": int(st.cycles), "rel_residual": float(st.rel_residual),
                     "kernel_launches_ms": dict(sorted(fam.items(), key=lambda kv: -kv[1][1]))}
    cuda.artss_mixed_destroy(mx)
    for h in mx_rb.values():
        cuda.artss_mixed_destroy(h)
    cuda.artss_mg_destroy(mg)
    ctx.close()
    ms = dist.max(res["mixed"]["ms_per_solve"])
    return {
        "metric": "ms per pressure solve to 1e-8 relative residual",
        "value": ms,
        "unit": "ms",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 V-cycles in f64 defect correction",
        "data": "synthetic",
        "config": {"workload": f"poisson_{n}cubed_neumann_boxes_{nl}levels", "cells": f"{n}x{n}x{n}",
                   "inner_cells": int(len(inner)), "boxes": len(sc.obstacles), "seed": args.seed,
                   "levels": nl, "rhs": "N(0,1) on fluid cells, zero mean, made consistent with the discrete operator (b = A p_inf, "
                          "relative change ~1e-4)", "start": "p = 0"},
        "plain_fp64": res["plain_fp64"],
        "mixed": res["mixed"],
        "mixed_rbgs_v11": res["mixed_rbgs_v11"],
        "mixed_rbgs_v22": res["mixed_rbgs_v22"],
        "speedup_vs_plain_fp64": res["plain_fp64"]["ms_per_solve"] / res["mixed"]["ms_per_solve"],
        "speedup_rbgs_vs_plain_fp64": {k: res["plain_fp64"]["ms_per_solve"] / res[k]["ms_per_solve"]
                                       for k in ("mixed_rbgs_v11", "mixed_rbgs_v22")},
    }


def run_ensemble(args, dist):
    """64 independent plume scenes of uneven grids (32-128 cells per axis), the
    mixed-precision pressure solve; scenes are split over the ranks by a
    greedy cell-count partition (no collective on the data path); on each GPU
    every scene runs in its own context and stream from its own host thread.
    value = all ranks' inner cells x steps / the slowest rank's device time."""
    import torch

    from artss_b200 import scenes
    from artss_b200.ensemble import Ensemble, partition

    torch.cuda.set_device(dist.local)
    scs = scenes.plume_ensemble(64, seed=args.seed, steps=args.warmup + args.steps + 4)
    cells = [sc.inner_cells() for sc in scs]
    mine = partition(cells, dist.world)[dist.rank]
    tmp = tempfile.mkdtemp(prefix="artss_ens_")
    # every scene's step is one graph launch from the third step on (captured in the warm-up)
    ens = Ensemble([scenes.write(scs[i], os.path.join(tmp, f"s{i}.xml")) for i in mine], device=dist.local,
                   graphs=True)
    ens.run(max(args.warmup, 3))
    streams = [torch.cuda.ExternalStream(s, device=torch.device("cuda", dist.local)) for s in ens.streams()]
    sampler = ClockSampler(dist.local)
    sampler.start()
    dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    start.record(streams[0] if streams else None)
    done = ens.run(args.steps)
    ends = []
    for st in streams:
        e = torch.cuda.Event(enable_timing=True)
        e.record(st)
        ends.append(e)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    ms = max((start.elapsed_time(e) for e in ends), default=0.0)
    assert all(d == args.steps for d in done), "a scene ended early"
    my_cells = float(ens.inner_cells) * args.steps
    graph_steps = sum(s.graph_steps for s in ens.sims)
    ens.close()
    ms_max = dist.max(ms)
    total = dist.sum(my_cells)
    return {
        "metric": "cell-updates/s per timestep (ensemble)",
        "value": total / (ms_max * 1e-3),
        "unit": "cell-updates/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64 (pressure: f32 V-cycles in f64 defect correction)",
        "data": "synthetic",
        "graph_steps": int(graph_steps),
        "config": {"workload": "plume_ensemble_64_scenes", "scenes": len(scs), "scenes_this_rank": len(mine),
                   "graphs": "whole-step CUDA graphs, 32 hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS)",
                   "inner_cells_total": int(sum(cells)), "sizes": [32, 48, 64, 96, 128], "dt": 0.005,
                   "pressure": "VCycleMGMixed to 1e-8 relative, at most 20 cycles per step",
                   "parallelism": f"scene partition over {dist.world} rank(s), one stream per scene"},
        "clocks": clocks,
        "e2e": None,
    }


def run_learned(args, dist):
    """ms per pressure solve to a 1e-8 relative residual inside time stepping
    (128x64x64 channel scenes of the ensemble family with 0-3 boxes): plain
    FP64 VCycleMG vs mixed precision vs learned guess + mixed precision, all
    from the previous step's pressure.  The network is trained first on
    samples the solver generates from other seeds (bounded budget, untimed)."""
    import numpy as np
    import torch

    from artss_b200 import learned as LN
    from artss_b200 import scenes

    torch.cuda.set_device(dist.local)
    dims = (64, 64, 128)
    tmp = tempfile.mkdtemp(prefix="artss_learned_")
    t0 = time.time()
    samples = LN.collect(range(100, 116), 16, 20, dims, tmp, device=dist.local, project=2)
    t1 = time.time()
    sc = LN.plume_channel(0, nx=dims[2], ny=dims[1], nz=dims[0])
    import artss_b200 as A
    sim = A.Simulation(scenes.write(sc, os.path.join(tmp, "net.xml")), device=dist.local)
    net = LN.UNet(sim.context, dims, seed=0)
    hist = LN.train(net, samples, epochs=4, lr=1e-3)
    t2 = time.time()
    res = LN.evaluate(net, [900 + 10 * dist.rank + k for k in range(2)], max(args.steps, 1), 20, dims, tmp,
                      device=dist.local, project=2, with_plain=True)
    sim.close()
    m = lambda k: float(np.mean(res[k]))  # noqa: E731
    learned_ms = dist.max(m("learned_ms"))
    return {
        "metric": "ms per pressure solve to 1e-8: learned vs plain MG",
        "value": learned_ms,
        "unit": "ms",
        "n_gpus": dist.world,
        "steps": len(res["learned_ms"]),
        "warmup": 20,
        "ms_per_step": learned_ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16 network (fp32 accumulation); f32 V-cycles in f64 defect correction",
        "data": "synthetic",
        "config": {"workload": "learned_guess_channel_128x64x64", "train_samples": len(samples), "epochs": 4,
                   "network": "3-level U-Net 16-32-64, 3x3x3 tcgen05 convolutions",
                   "guess": "p_prev + coarse-projected (2 levels) network correction, fallback to p_prev "
                            "when its initial residual is larger"},
        "plain_fp64": {"ms_per_solve": m("plain_ms"), "cycles": m("plain_cycles")},
        "mixed_from_p_prev": {"ms_per_solve": m("baseline_ms"), "cycles": m("baseline_cycles")},
        "learned_plus_mixed": {"ms_per_solve": m("learned_ms"), "cycles": m("learned_cycles"),
                               "inference_ms": m("infer_ms"), "fallbacks": res["fallbacks"],
                               "guess_residual_over_p_prev_residual": m("residual_ratio")},
        "speedup_vs_plain_fp64": m("plain_ms") / m("learned_ms"),
        "note": ("the network's guess was discarded (fallback to p_prev) on %d of %d solves; the cycles saved "
                 "against plain FP64 come from the mixed-precision solver" % (res["fallbacks"], len(res["learned_ms"]))),
        "l2": "flushed (256 MB written) before every timed solve",
        "training": {"collect_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1),
                     "loss_per_epoch": [round(h, 4) for h in hist]},
    }


def cpu_baseline(args, inner):
    """The reference serial build (oracle/_ref) on a bounded sample of the same
    workload: the first steps of the same scene, steady-state steps timed."""
    from tests import refdriver
    if not refdriver.available():
        return None
    name, sc = workload(args.workload, args.cpu_steps, args.channel_nx)
    tmp = tempfile.mkdtemp(prefix="artss_cpu_")
    from artss_b200 import scenes
    xml = scenes.write(sc, os.path.join(tmp, f"{name}_cpu.xml"))
    t = refdriver.timing(xml, args.cpu_steps)
    steady = t["step_ms"][1:] or t["step_ms"]
    value = t["inner_cells"] * len(steady) / (sum(steady) * 1e-3)
    return {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
            "sample": f"{args.cpu_steps} steps of the same scene with the unmodified ARTSS serial build "
                      f"(g++ -O3, one core); steps 2..{args.cpu_steps} timed, step 1 (first-step pressure solve "
                      f"to tolerance) {t['step_ms'][0]:.0f} ms excluded like the GPU warm-up"}


def run_reference(args, dist):
    """--impl reference: the reference serial build, rank 0 only."""
    from tests import refdriver
    name, sc = workload(args.workload, args.warmup + args.steps, args.channel_nx)
    if not refdriver.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/artss_ref_driver is not built (make -C oracle ref)"}
    from artss_b200 import scenes
    tmp = tempfile.mkdtemp(prefix="artss_ref_")
    xml = scenes.write(sc, os.path.join(tmp, f"{name}_ref.xml"))
    t = refdriver.timing(xml, args.warmup + args.steps, timeout=7200)
    timed = t["step_ms"][args.warmup:args.warmup + args.steps]
    ms = sum(timed)
    value = t["inner_cells"] * len(timed) / (ms * 1e-3)
    return {
        "impl": "reference",
        "metric": "cell-updates/s per timestep",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": dist.world,
        "steps": len(timed),
        "warmup": args.warmup,
        "ms_per_step": ms / max(len(timed), 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": step_config(name, sc, t["inner_cells"], dist.world),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"{args.warmup} warm-up + {len(timed)} timed steps of the unmodified ARTSS "
                                   "serial build (it has no multi-threaded CPU path; its OpenACC multicore build "
                                   "needs NVHPC, absent here)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    if args.workload == "ensemble":
        # scenes run on their own streams: give them 32 hardware work queues
        # instead of the default 8 (read when the CUDA context is created)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    dist = Dist()
    try:
        if args.impl == "reference":
            if dist.rank == 0:
                print(json.dumps(run_reference(args, dist)), flush=True)
            return
        if args.workload in ("poisson", "ensemble", "learned"):
            out = {"poisson": run_poisson, "ensemble": run_ensemble, "learned": run_learned}[args.workload](args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
            return
        out, xml, inner = run_b200(args, dist)
        if dist.rank == 0:
            if dist.world == 1 and not args.no_cpu_baseline:
                out["cpu_baseline"] = cpu_baseline(args, inner)
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
