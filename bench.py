"""Benchmark: body-steps/s of the device contact pipeline on the 100,000-body
mixed-shape scene (spheres, boxes, capsules, cylinders, 16-vertex hulls in a
200 x 200 x 60 m box above a plane; dt = 1/60 s, 4 substeps), seeded synthetic
data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --workload batched [--steps K] ...   (4096 independent worlds)

b200 arm: one process per GPU (torchrun for N > 1); every rank steps its own
replica of the world ("replicas only": a single world does not shard), the
timed region is K steps on the device (CUDA events on the pipeline's stream,
L2 flushed with a 256 MiB write before every step, outside the events), and
the value is all ranks' bodies x steps / max-over-ranks time.

reference arm: the reference engine's CPU backend (built from its sources
into oracle/_ref), all host cores, on the same scene; rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-steps/s @100k bodies"
DT = 1.0 / 60.0
CONFIG = 2            # the 100k-body mixed-shape scene
SUBSTEPS = 4
L2_FLUSH_BYTES = 256 << 20

# Roofline of the narrow phase's neighbour, the island solve: algorithmic bytes
# per contact row and sweep (contact constants 64 + impulses r/w 48 + two
# bodies' pose/velocity/mass reads 168 + velocity writes 48).
SOLVER_BYTES_PER_ROW = 328
# Rewind: one distance query reads both bodies' 256-byte records.
REWIND_BYTES_PER_QUERY = 512
# Memory-bound stages: (stage, algorithmic bytes per body, per candidate pair).
# prepare: velocity integration 60 + pose copy 56; broadphase: AABB 72, keys
# 44, cell table 12, neighbour search 36 per body + 8 per emitted pair;
# cell_sort: 4 passes x (8 + 4) B read and written per body.
MEMORY_STAGE_BYTES = [("prepare", 116, 0), ("broadphase", 164, 8), ("cell_sort", 96, 0)]
# DRAM bytes per step of the same stages on the 100,001-body scene: the sum of
# their kernels' dram__bytes_read.sum + dram__bytes_write.sum per launch from
# one ncu capture each (writes stay in L2 within a launch).
MEMORY_STAGE_TRAFFIC = {"prepare": 16.02e6, "broadphase": 11.21e6 + 4.81e6 + 2.78e6 + 9.16e6}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_scene(size):
    import velox_b200 as vb
    specs, pool = vb.generate_scene(CONFIG, seed=CONFIG, size=size)
    bodies, hull, faces = vb.bodies_from_specs(specs, pool)
    return specs, pool, bodies, vb.make_soup(hull, faces)


def cpu_baseline(specs, pool, n_bodies, checkpoints, total_steps):
    """The reference CPU backend (default Release build, all host threads) on
    the same scene, sampled along the trajectory: from each checkpoint state
    (captured during the timed device steps, evenly spaced), one step to settle
    the contact caches and one timed step. Each timed step stands for its
    share of the trajectory, so early cheap steps and late pile steps weigh
    what they weigh in the device run."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available(strict=False):
        return None
    w = ref.RefWorld(specs, pool, backend=ref.BACKEND_CPU, strict=False)
    w.configure(substeps=SUBSTEPS, workers=0)
    workers = int(w.L.ref_world_worker_count(w.h))
    est, spent = 0.0, 0.0
    t0 = time.perf_counter()
    for state in checkpoints:
        w.set_bodies(state)
        w.step(DT, 1)
        est += (w.step(DT, 1) / 1000.0) * (total_steps / len(checkpoints))
    spent = time.perf_counter() - t0
    single = one_worker_sample(w, n_bodies, budget_s=10.0, max_steps=2)
    w.close()
    value = n_bodies * total_steps / est
    return {"value": value, "unit": "body-steps/s", "cores": workers, "kind": "reference",
            "single_worker": single,
            "sample": f"{len(checkpoints)} timed steps of the {n_bodies}-body scene, one from each of "
                      f"{len(checkpoints)} evenly spaced states of the {total_steps}-step device trajectory "
                      f"(each after one settling step), weighted equally; reference CPU backend (Release "
                      f"build), {workers} worker threads on {os.cpu_count()} host cores; {spent:.1f} s"}


def single_config(n, world):
    """The workload description both arms print (identical for the same N)."""
    return {"workload": f"mixed-shape scene, {n} bodies (1 plane), dt 1/60 s, {SUBSTEPS} substeps",
            "bodies": n, "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MiB write) before every timed step, outside the step's events"}


def one_worker_sample(w, n, budget_s=20.0, max_steps=3):
    """The reference CPU backend with setWorkerCount(1) on the world's current
    state: up to `max_steps` steps within `budget_s`."""
    w.configure(substeps=SUBSTEPS, workers=1)
    steps, total = 0, 0.0
    while steps < max_steps and total < budget_s:
        total += w.step(DT, 1) / 1000.0
        steps += 1
    return {"value": n * steps / total, "unit": "body-steps/s", "cores": 1, "kind": "reference",
            "sample": f"{steps} steps continuing the same trajectory, reference CPU backend (Release build), "
                      f"setWorkerCount(1)"}


def run_reference(args):
    """The reference CPU backend (built from its sources into oracle/_ref) on
    the same scene. The scene specs come from the generator compiled into that
    build, so this process loads no library of this package."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    budget = float(os.environ.get("VXB_REFERENCE_BUDGET_S", "240"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available(strict=False):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}))
        return 0
    specs, pool = ref.generate_scene(CONFIG, seed=CONFIG, size=args.size)
    n = len(specs)
    w = ref.RefWorld(specs, pool, backend=ref.BACKEND_CPU, strict=False)
    w.configure(substeps=SUBSTEPS, workers=0)
    workers = int(w.L.ref_world_worker_count(w.h))
    w.step(DT, args.warmup)
    steps, total = 0, 0.0
    while steps < args.steps and total < budget:
        total += w.step(DT, 1) / 1000.0
        steps += 1
    single = one_worker_sample(w, n)
    w.close()
    value = n * steps / total
    sample = (f"{steps} of {args.steps} requested steps (time budget {budget:.0f} s) of the {n}-body scene after "
              f"{args.warmup} warm-up steps; reference CPU backend (Release build), {workers} worker threads on "
              f"{os.cpu_count()} host cores")
    line = {"metric": METRIC, "value": value, "unit": "body-steps/s", "impl": "reference", "n_gpus": 0,
            "steps": steps, "warmup": args.warmup, "ms_per_step": total / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": single_config(n, world),
            "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": workers, "kind": "reference",
                             "sample": sample, "single_worker": single},
            "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


BATCH_CONFIG = 4      # independent worlds: plane + log-uniform [8, 512] spheres/boxes/capsules each
PLAIN_SAMPLE = 48     # worlds stepped one at a time for the plain comparison
CPU_SAMPLE = 48       # worlds stepped by the reference CPU backend


def run_batched(args):
    """world-steps/s of 4096 independent worlds packed into one context (world
    id in the cell-key high bits, islands never cross worlds), next to the
    same worlds stepped one world per context (the plain single-world path:
    a sample of worlds spread over the size distribution, scaled by their
    share of the batch) and the reference CPU backend on a sample of worlds.
    Under torchrun the worlds are split across ranks (strong scaling, no
    data-path collective)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nworlds = args.size if args.size != 100000 else 4096
    if args.impl == "reference":
        if rank != 0:
            return 0
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref
        if not ref.available(strict=False):
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}))
            return 0
        specs, pool = ref.generate_scene(BATCH_CONFIG, seed=BATCH_CONFIG, size=nworlds)
        return run_batched_reference(args, specs, pool, nworlds)
    import torch
    import velox_b200 as vb
    from velox_b200.ranks import max_over_ranks, shard_specs

    specs, pool = vb.generate_scene(BATCH_CONFIG, seed=BATCH_CONFIG, size=nworlds)
    mine, lo, hi = shard_specs(specs, nworlds, rank, world)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    bodies, hull, faces = vb.bodies_from_specs(mine, pool)
    soup = vb.make_soup(hull, faces)
    worlds_here = hi - lo
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(ctx, steps, host=None):
        events = []
        with torch.cuda.stream(stream):
            for _ in range(steps):
                flush.fill_(1)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if host:
                    ctx.write_forces(host[0])
                ctx.step(1)
                if host:
                    ctx.read_poses(host[1])
                e1.record(stream)
                events.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in events)

    # batched
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.load(bodies, soup, world_of=mine["world"])
    ctx.configure(dt=DT, substeps=SUBSTEPS)
    ctx.step(max(args.warmup, 3))
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    launches0 = ctx.launches
    syncs0 = ctx.host_syncs
    ctx.enable_timing(True)
    if args.profile:
        torch.cuda.cudart().cudaProfilerStart()
    ms = timed(ctx, args.steps)
    if args.profile:
        torch.cuda.cudart().cudaProfilerStop()
    barrier()
    clocks = sampler.stop()
    launches = ctx.launches - launches0
    host_syncs = ctx.host_syncs - syncs0
    stage = ctx.stage_times()
    last = ctx.stats()
    ctx.close()
    ms = max_over_ranks(ms, dist, "cuda")
    value = nworlds * args.steps / (ms / 1e3)

    # e2e: a fresh batched world through the C ABI with host buffers every step
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.load(bodies, soup, world_of=mine["world"])
    ctx.configure(dt=DT, substeps=SUBSTEPS)
    ctx.step(max(args.warmup, 3))
    n = len(bodies)
    forces = torch.zeros((n, 6), dtype=torch.float32).pin_memory()
    poses = torch.zeros((n, 7), dtype=torch.float32).pin_memory()
    barrier()
    e2e_ms = timed(ctx, args.steps, (forces.numpy(), poses.numpy()))
    ctx.close()
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")

    # plain: sampled worlds one per context, scaled by their body share
    plain = None
    if rank == 0 and not args.profile:
        counts = np.bincount(specs["world"], minlength=nworlds)
        order = np.argsort(counts, kind="stable")
        sample = order[np.linspace(0, nworlds - 1, min(PLAIN_SAMPLE, nworlds)).astype(int)]
        total_ms = 0.0
        for w in sample:
            one = specs[specs["world"] == w].copy()
            one["world"] = 0
            b1, h1, f1 = vb.bodies_from_specs(one, pool)
            c1 = vb.Context(local)
            c1.set_stream(stream.cuda_stream)
            c1.load(b1, vb.make_soup(h1, f1))
            c1.configure(dt=DT, substeps=SUBSTEPS)
            c1.step(max(args.warmup, 3))
            total_ms += timed(c1, args.steps)
            c1.close()
        per_world_ms = total_ms / len(sample) / args.steps
        plain = {"value": 1e3 / per_world_ms, "unit": "world-steps/s",
                 "sample": f"{len(sample)} worlds spread over the body-count distribution, each in its own context, "
                           f"{args.steps} device-timed steps after {max(args.warmup, 3)} warm-up steps; "
                           f"one world at a time on this GPU"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and not args.profile:
        try:
            cpu = batched_cpu_baseline(specs, pool, nworlds, min(args.steps, 20))
        except Exception as exc:  # reported, not fatal
            cpu = {"error": str(exc)}
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    bodies_total = int(len(specs))
    line = {"metric": f"world-steps/s @{nworlds} worlds", "value": value, "unit": "world-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{nworlds} independent worlds, plane + log-uniform [8,512] spheres/boxes/capsules "
                                   f"each ({bodies_total} bodies), dt 1/60 s, {SUBSTEPS} substeps",
                       "worlds": nworlds, "bodies": bodies_total, "parallelism": f"worlds split over {world} GPU(s)",
                       "l2": "flushed (256 MiB write) before every timed step, outside the step's events"},
            "body_steps_per_s": bodies_total * args.steps / (ms / 1e3),
            "plain": plain, "vs_plain": value / plain["value"] if plain else None,
            "last_step": last, "stage_ms_per_step": {k: v[0] / args.steps for k, v in stage.items()},
            "cpu_baseline": cpu,
            "e2e": {"value": nworlds * args.steps / (e2e_ms / 1e3), "unit": "world-steps/s",
                    "h2d_bytes_per_step": int(forces.numel() * 4), "d2h_bytes_per_step": int(poses.numel() * 4)},
            "clocks": clocks, "gpu_launches": int(launches), "host_syncs_per_step": host_syncs / args.steps}
    print(json.dumps(line))
    return 0


def batched_cpu_baseline(specs, pool, nworlds, steps):
    """Reference CPU backend (Release build, all host threads) on sampled worlds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available(strict=False):
        return None
    counts = np.bincount(specs["world"], minlength=nworlds)
    order = np.argsort(counts, kind="stable")
    sample = order[np.linspace(0, nworlds - 1, min(CPU_SAMPLE, nworlds)).astype(int)]
    total = 0.0
    workers = 0
    for w in sample:
        one = specs[specs["world"] == w].copy()
        one["world"] = 0
        rw = ref.RefWorld(one, pool, backend=ref.BACKEND_CPU, strict=False)
        rw.configure(substeps=SUBSTEPS, workers=0)
        workers = int(rw.L.ref_world_worker_count(rw.h))
        rw.step(DT, 3)
        for _ in range(steps):
            total += rw.step(DT, 1) / 1000.0
        rw.close()
    value = len(sample) * steps / total
    return {"value": value, "unit": "world-steps/s", "cores": workers, "kind": "reference",
            "sample": f"{len(sample)} worlds spread over the body-count distribution, {steps} steps each after 3 "
                      f"warm-up steps, one world at a time; reference CPU backend (Release build), {workers} worker "
                      f"threads on {os.cpu_count()} host cores"}


def run_batched_reference(args, specs, pool, nworlds):
    cpu = batched_cpu_baseline(specs, pool, nworlds, min(args.steps, 20))
    if cpu is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) missing"}))
        return 0
    line = {"metric": f"world-steps/s @{nworlds} worlds", "value": cpu["value"], "unit": "world-steps/s",
            "impl": "reference", "n_gpus": 0, "steps": min(args.steps, 20), "warmup": 3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": f"{nworlds} independent worlds (sampled)", "worlds": nworlds},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "world-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=100000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the reference CUDA backend and the batched, adjoint and stacking workloads "
                         "reported beside the headline")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (ncu --profile-from-start off)")
    ap.add_argument("--workload", default="single", choices=["single", "batched"],
                    help="single: the 100k-body world (default); batched: 4096 independent worlds in one context")
    args = ap.parse_args()
    if args.workload == "batched":
        return run_batched(args)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import velox_b200 as vb
    from velox_b200.ranks import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    specs, pool, bodies, soup = build_scene(args.size)
    n = len(bodies)
    stream = torch.cuda.Stream()
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.load(bodies, soup)
    ctx.configure(dt=DT, substeps=SUBSTEPS)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    ctx.step(max(args.warmup, 3) if args.warmup >= 3 else args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    launches0 = ctx.launches
    syncs0 = ctx.host_syncs
    ctx.enable_timing(True)
    events = []
    contacts_total = 0
    gap_queries_total = 0
    pairs_total = 0
    chain_us = 0
    if args.profile:
        torch.cuda.cudart().cudaProfilerStart()
    checkpoints = []
    marks = {int(args.steps * i / 5) for i in range(5)}
    with torch.cuda.stream(stream):
        for step in range(args.steps):
            if step in marks and rank == 0 and world == 1 and not args.no_cpu_baseline:
                checkpoints.append(ctx.read_bodies())  # between steps, outside the events
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.step(1)
            e1.record(stream)
            events.append((e0, e1))
            st = ctx.stats()
            contacts_total += st["contacts"]
            gap_queries_total += st["rewindGapQueries"]
            pairs_total += st["candidatePairs"]
            chain_us += st["rewindSpeculateMicros"] + st["rewindCriticalMicros"]
    if args.profile:
        torch.cuda.cudart().cudaProfilerStop()
    barrier()
    clocks = sampler.stop()
    launches = ctx.launches - launches0
    host_syncs = ctx.host_syncs - syncs0
    stage = ctx.stage_times()
    ctx.enable_timing(False)
    ms = sum(a.elapsed_time(b) for a, b in events)
    ms = max_over_ranks(ms, dist, "cuda")
    value = world * n * args.steps / (ms / 1e3)

    # Roofline. Island solve: memory-bound sweeps over contact rows.
    # Rewind: distance queries on two bodies' records along a dependency
    # chain (latency-bound; reported against the same HBM peak).
    peak, peak_kind = measured_peaks()
    solve_ms, solve_calls = stage["solve"]
    rows = contacts_total * 2 * 8 * SUBSTEPS  # sweeps * substeps per step
    solve_bytes = rows * SOLVER_BYTES_PER_ROW
    solve_gbs = solve_bytes / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    solve_roofline = {"bound": "hbm", "kernel": "solveTinyKernel+solveBlockKernel+solveClusterKernel (substep solve)",
                      "achieved": solve_gbs, "peak": peak, "unit": "GB/s", "frac": solve_gbs / peak,
                      "peak_source": peak_kind, "traffic": None,
                      "algorithmic_bytes_per_launch": solve_bytes / max(solve_calls, 1),
                      "avg_launch_ms": solve_ms / max(solve_calls, 1)}
    rewind_ms, rewind_calls = stage["rewind"]
    rewind_bytes = gap_queries_total * REWIND_BYTES_PER_QUERY
    rewind_gbs = rewind_bytes / (rewind_ms / 1e3) / 1e9 if rewind_ms > 0 else 0.0
    rewind_roofline = {"bound": "hbm", "kernel": "caProbeKernel+caFlowKernel (rewind pass)",
                       "achieved": rewind_gbs, "peak": peak, "unit": "GB/s", "frac": rewind_gbs / peak,
                       "peak_source": peak_kind, "traffic": None,
                       "algorithmic_bytes_per_launch": rewind_bytes / max(rewind_calls, 1),
                       "avg_launch_ms": rewind_ms / max(rewind_calls, 1),
                       # the pass's own dependency chain: the longest single pair's
                       # conservative advancement (speculated in parallel) plus the
                       # longest chain of the ordered pass
                       "chain_ms_per_step": chain_us / 1e3 / args.steps,
                       "chain_frac": (chain_us / 1e3) / rewind_ms if rewind_ms > 0 else None,
                       "note": "a chain of dependent distance queries: latency-bound, not bandwidth-bound"}
    # Memory-bound stages: algorithmic bytes per step (the per-unit figures in
    # MEMORY_STAGE_BYTES) over the stage's own CUDA-event time.
    memory_rooflines = []
    for name, per_body, per_pair in MEMORY_STAGE_BYTES:
        st_ms, st_calls = stage[name]
        if st_ms <= 0:
            continue
        algo = per_body * n * args.steps + per_pair * pairs_total
        gbs = algo / (st_ms / 1e3) / 1e9
        memory_rooflines.append({"stage": name, "bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                 "frac": gbs / peak, "peak_source": peak_kind,
                                 "algorithmic_bytes_per_step": algo / args.steps,
                                 "ms_per_step": st_ms / args.steps,
                                 "traffic": MEMORY_STAGE_TRAFFIC.get(name)})
    dominant = max(stage.items(), key=lambda kv: kv[1][0])[0]
    roofline = rewind_roofline if dominant == "rewind" else solve_roofline
    roofline = dict(roofline, stage=dominant)

    # End to end through the C ABI, on a fresh world over the same steps:
    # forces in from pinned host memory, one step, poses back to pinned host
    # memory, every step (host copies inside the timed region).
    ctx2 = vb.Context(local)
    ctx2.set_stream(stream.cuda_stream)
    ctx2.load(bodies, soup)
    ctx2.configure(dt=DT, substeps=SUBSTEPS)
    ctx2.step(max(args.warmup, 3) if args.warmup >= 3 else args.warmup)
    forces = torch.zeros((n, 6), dtype=torch.float32).pin_memory()
    poses = torch.zeros((n, 7), dtype=torch.float32).pin_memory()
    fptr, pptr = forces.numpy(), poses.numpy()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        ctx2.write_forces(fptr)
        ctx2.step(1)
        ctx2.read_poses(pptr)
    e1.record(stream)
    barrier()
    wall = time.perf_counter() - t0
    ctx2.close()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    e2e = {"value": world * n * args.steps / (e2e_ms / 1e3), "unit": "body-steps/s",
           "h2d_bytes_per_step": int(forces.numel() * 4), "d2h_bytes_per_step": int(poses.numel() * 4),
           "steps": args.steps, "wall_s": wall}

    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            baseline = cpu_baseline(specs, pool, n, checkpoints, args.steps)
        except Exception as exc:  # reported, not fatal
            baseline = {"error": str(exc)}

    plain_gpu = None
    if rank == 0 and world == 1 and not args.no_extras and not args.profile:
        try:
            plain_gpu = reference_gpu(specs, pool, n, args.steps, max(args.warmup, 3))
            if plain_gpu and "value" in plain_gpu:
                plain_gpu["e2e_vs_plain_gpu"] = e2e["value"] / plain_gpu["value"]
        except Exception as exc:  # reported, not fatal
            plain_gpu = {"error": str(exc)}

    stats = ctx.stats()
    autotune = tuned_shapes(ctx)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    extra = {}
    if world == 1 and not args.no_extras and not args.profile:
        extra = run_extras(args, local, stream)
    line = {"metric": METRIC, "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": single_config(n, world),
            "contacts_per_s": contacts_total / (ms / 1e3), "last_step": stats,
            "stage_ms_per_step": {k: v[0] / args.steps for k, v in stage.items()},
            "roofline": roofline, "solve_roofline": solve_roofline, "rewind_roofline": rewind_roofline,
            "memory_rooflines": memory_rooflines,
            "cpu_baseline": baseline, "e2e": e2e, "clocks": clocks,
            "gpu_launches": int(launches), "host_syncs_per_step": host_syncs / args.steps,
            "autotune": autotune, "plain_gpu": plain_gpu}
    line.update(extra)
    print(json.dumps(line))
    return 0


def tuned_shapes(ctx):
    """Launch shapes the tuner decided, per site and size bucket
    (floor(log2(items)) -> [threads, blocks per SM])."""
    out = {}
    for site in ("collide_convex", "collide_plane", "rewind_probe"):
        decided = {}
        for bucket in range(4, 25):
            threads, per_sm, done = ctx.tuned_shape(site, 1 << bucket)
            if done:
                decided[str(bucket)] = [threads, per_sm]
        out[site] = decided
    return out


def reference_gpu(specs, pool, n, steps, warmup, budget_s=60.0):
    """The reference's own CUDA backend (src/backend_cuda.cu built for sm_100a
    with its default flags, World(BackendType::Cuda)) on the same scene and
    this GPU: the plain single-world GPU path. Its World::step is blocking
    (host copies every step), so the per-step time is the host wall time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available("cuda_fast"):
        return None
    w = ref.RefWorld(specs, pool, backend=ref.BACKEND_CUDA_EMULATED, strict="cuda_fast")
    if w.L.ref_world_backend_name(w.h) != b"cuda":
        w.close()
        return {"error": "reference CUDA backend unavailable on this device"}
    w.configure(substeps=SUBSTEPS, workers=0)
    w.step(DT, warmup)
    done, total = 0, 0.0
    while done < steps and total < budget_s:
        total += w.step(DT, 1) / 1000.0
        done += 1
    w.close()
    return {"value": n * done / total, "unit": "body-steps/s", "steps": done, "ms_per_step": total / done * 1e3,
            "kind": "reference CUDA backend (src/backend_cuda.cu, sm_100a, default flags) on this GPU",
            "timing": "host wall time of World::step (blocking), after the same warm-up"}


# ---- the other workloads, reported beside the headline -----------------------

STACK_CONFIG = 3      # 256 twenty-row box pyramids, 8 substeps, 600 steps
ADJOINT_CONFIG = 5    # 1024 worlds: 5-box stack + sphere projectile, 120 steps, checkpoints every 10


def _timed_blocks(ctx, stream, flush, steps, block=1):
    """Device time of `steps` steps in blocks of `block` (L2 flushed before each block)."""
    import torch
    events = []
    with torch.cuda.stream(stream):
        done = 0
        while done < steps:
            k = min(block, steps - done)
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.step(k)
            e1.record(stream)
            events.append((e0, e1))
            done += k
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in events)


def measure_batched(local, stream, nworlds, steps, warmup, plain_sample=PLAIN_SAMPLE):
    """world-steps/s of `nworlds` independent worlds in one context, next to
    the same worlds stepped one world at a time: in this library (one context
    per world) and on the reference's own CUDA backend (one World per world)."""
    import torch
    import velox_b200 as vb
    specs, pool = vb.generate_scene(BATCH_CONFIG, seed=BATCH_CONFIG, size=nworlds)
    bodies, hull, faces = vb.bodies_from_specs(specs, pool)
    soup = vb.make_soup(hull, faces)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.load(bodies, soup, world_of=specs["world"])
    ctx.configure(dt=DT, substeps=SUBSTEPS)
    ctx.step(max(warmup, 3))
    torch.cuda.synchronize()
    launches0, syncs0 = ctx.launches, ctx.host_syncs
    ms = _timed_blocks(ctx, stream, flush, steps)
    launches, syncs = ctx.launches - launches0, ctx.host_syncs - syncs0
    ctx.close()
    value = nworlds * steps / (ms / 1e3)
    counts = np.bincount(specs["world"], minlength=nworlds)
    order = np.argsort(counts, kind="stable")
    sample = order[np.linspace(0, nworlds - 1, min(plain_sample, nworlds)).astype(int)]
    total_ms = 0.0
    for w in sample:
        one = specs[specs["world"] == w].copy()
        one["world"] = 0
        b1, h1, f1 = vb.bodies_from_specs(one, pool)
        c1 = vb.Context(local)
        c1.set_stream(stream.cuda_stream)
        c1.load(b1, vb.make_soup(h1, f1))
        c1.configure(dt=DT, substeps=SUBSTEPS)
        c1.step(max(warmup, 3))
        torch.cuda.synchronize()
        total_ms += _timed_blocks(c1, stream, flush, steps)
        c1.close()
    plain = 1e3 / (total_ms / len(sample) / steps)
    plain_ref = None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if ref.available("cuda_fast"):
        ref_s, ref_steps = 0.0, 0
        for w in sample:
            one = specs[specs["world"] == w].copy()
            one["world"] = 0
            rw = ref.RefWorld(one, pool, backend=ref.BACKEND_CUDA_EMULATED, strict="cuda_fast")
            rw.configure(substeps=SUBSTEPS, workers=0)
            rw.step(DT, max(warmup, 3))
            for _ in range(steps):
                ref_s += rw.step(DT, 1) / 1000.0
                ref_steps += 1
            rw.close()
        plain_ref = {"value": ref_steps / ref_s, "unit": "world-steps/s",
                     "kind": "reference CUDA backend (src/backend_cuda.cu, sm_100a), one World per world, stepped "
                             "one world at a time on this GPU (host wall time of the blocking World::step)",
                     "sample": f"{len(sample)} worlds over the body-count distribution, {steps} steps each"}
    return {"metric": f"world-steps/s @{nworlds} worlds", "value": value, "unit": "world-steps/s",
            "steps": steps, "warmup": max(warmup, 3), "ms_per_step": ms / steps,
            "bodies": int(len(specs)), "body_steps_per_s": len(specs) * steps / (ms / 1e3),
            "workload": f"{nworlds} independent worlds, plane + log-uniform [8,512] spheres/boxes/capsules each "
                        f"({len(specs)} bodies), dt 1/60 s, {SUBSTEPS} substeps",
            "plain": {"value": plain, "unit": "world-steps/s",
                      "sample": f"{len(sample)} worlds over the body-count distribution, one context per world, "
                                f"one world at a time, {steps} device-timed steps each"},
            "vs_plain": value / plain, "gpu_launches": int(launches), "host_syncs_per_step": syncs / steps,
            "plain_reference_gpu": plain_ref,
            "vs_plain_reference_gpu": value / plain_ref["value"] if plain_ref else None}


def measure_adjoint(local, stream, nworlds=1024, steps=120, every=10):
    """The differentiation workload: forward with the tape, and the backward
    pass (vxb_adjoint_backward) over the same steps; adjoint/forward time."""
    import torch
    import velox_b200 as vb
    specs, pool = vb.generate_scene(ADJOINT_CONFIG, seed=ADJOINT_CONFIG, size=nworlds)
    bodies, hull, faces = vb.bodies_from_specs(specs, pool)
    soup = vb.make_soup(hull, faces)
    world_of = np.ascontiguousarray(specs["world"], np.uint32)
    boxes = bodies["shape"] == vb.binding.SHAPE["box"]
    rng = np.random.default_rng(ADJOINT_CONFIG)
    target = np.zeros((len(bodies), 3), np.float32)
    target[boxes] = rng.normal(scale=0.05, size=(int(boxes.sum()), 3))
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)

    def forward(tape):
        ctx.load(bodies, soup, world_of=world_of)
        ctx.configure(dt=DT, substeps=SUBSTEPS)
        if tape:
            ctx.tape_begin(steps, every)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    forward(True)  # warm-up (allocations, module loading)
    fwd_plain = forward(False)
    fwd_tape = forward(True)
    final = ctx.read_bodies()
    d = final["position"] - bodies["position"] - target
    seed = np.zeros((len(bodies), 13), np.float32)
    seed[boxes, 0:3] = 2.0 * d[boxes]
    ctx.adjoint_backward(seed)  # warm-up
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    grad, ginv, gmass, flags = ctx.adjoint_backward(seed)
    e1.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    bwd = e0.elapsed_time(e1)
    ctx.close()
    sphere = bodies["shape"] == vb.binding.SHAPE["sphere"]
    return {"metric": "adjoint/forward time", "value": bwd / fwd_tape, "unit": "ratio", "higher_is_better": False,
            "workload": f"{nworlds} worlds, 5-box stack + sphere projectile each ({len(bodies)} bodies), "
                        f"{steps} steps, dt 1/60 s, {SUBSTEPS} substeps, checkpoints every {every} steps",
            "forward_ms": fwd_tape, "forward_untaped_ms": fwd_plain, "backward_ms": bwd,
            "backward_wall_ms": wall_ms, "vs_untaped_forward": bwd / fwd_plain,
            "smooth_worlds": int(np.sum(flags == 0)), "worlds": nworlds,
            "rewound_worlds": int(np.sum((flags & 1) != 0)), "diverged_worlds": int(np.sum((flags & 2) != 0)),
            "loss": float(np.sum(d[boxes] ** 2)),
            "grad_norm": {"sphere_velocity": float(np.linalg.norm(grad[sphere, 7:10])),
                          "sphere_angular_velocity": float(np.linalg.norm(grad[sphere, 10:13])),
                          "mass": float(np.linalg.norm(gmass))}}


def measure_stacking(local, stream, pyramids=256, steps=600, block=100):
    """Solver-heavy stacking: 256 twenty-row box pyramids (53,760 boxes),
    8 substeps, 600 steps; pass = every pyramid standing and no contact deeper
    than 5 mm (sampled every `block` steps)."""
    import torch
    import velox_b200 as vb
    specs, pool = vb.generate_scene(STACK_CONFIG, seed=STACK_CONFIG, size=pyramids)
    bodies, hull, faces = vb.bodies_from_specs(specs, pool)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ctx = vb.Context(local)
    ctx.set_stream(stream.cuda_stream)
    ctx.load(bodies, vb.make_soup(hull, faces))
    ctx.configure(dt=DT, substeps=8)
    start = bodies["position"].copy()
    ms, deepest = 0.0, 0.0
    for _ in range(steps // block):
        ms += _timed_blocks(ctx, stream, flush, block, block)
        contacts = ctx.read_contacts()
        deepest = min(deepest, float(contacts["gap"].min()) if len(contacts) else 0.0)
    end = ctx.read_bodies()["position"]
    ctx.close()
    drift = end[1:] - start[1:]
    standing = bool(np.abs(drift[:, 1]).max() < 0.05 and np.linalg.norm(drift, axis=1).max() < 0.1)
    n = len(bodies) - 1
    return {"metric": f"body-steps/s @{n} stacked boxes", "value": n * steps / (ms / 1e3), "unit": "body-steps/s",
            "workload": f"{pyramids} twenty-row box pyramids ({n} boxes), friction 0.6, dt 1/60 s, 8 substeps",
            "steps": steps, "ms_per_step": ms / steps, "max_penetration_m": -deepest,
            "max_drift_m": float(np.linalg.norm(drift, axis=1).max()), "all_standing": standing,
            "pass": standing and deepest >= -5e-3,
            "l2": f"flushed before every {block}-step block"}


def run_extras(args, local, stream):
    out = {}
    for name, fn in [("batched", lambda: measure_batched(local, stream, 4096, min(args.steps, 20), args.warmup)),
                     ("adjoint", lambda: measure_adjoint(local, stream)),
                     ("stacking", lambda: measure_stacking(local, stream))]:
        try:
            out[name] = fn()
        except Exception as exc:  # reported, not fatal
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


if __name__ == "__main__":
    sys.exit(main())
