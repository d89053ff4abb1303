#!/usr/bin/env python3
# SPDX-License-Identifier: MIT
"""Benchmark: steps/sec of the 65,536-box pile at equal residual.

Workload: box_pile((64, 32, 32), seed=4) -- 65,536 random boxes (edges
U[0.5,1.5] m, density U[500,2000] kg/m^3, friction U[0.3,0.8]) plus a static
ground and four walls -- starting from the settled state in
tests/golden/settled_pile_64x32x32.npz (300 ticks of plain AVBD from the spawn
grid). A step is one rigid AVBD tick (legacy profile: predict, broadphase,
narrowphase, contact cache, prepare, colouring, solve, impact phase, commit)
run with the residual-driven schedule: sweep until the position violation of
the active contact normal rows and hard joint rows is within --tolerance (1e-4
m), at most --max-iterations sweeps. --residual-norm picks how the rows are
judged: `p999` (default) stops once at most one row in a thousand violates by
more than the tolerance; `max` once every row is within it (on this pile the
largest row violation levels off at 2-5e-4 m and no sweep count reaches 1e-4
m, so both arms would run to the cap); `rms` once the RMS is within it (met
after about 4 sweeps while single rows still violate by millimetres). Each
arm's largest row violation, RMS and violating fraction are reported. Inputs
are synthetic (seeded); no dataset is involved.

GPU arm (default): the warm-start MLP is first trained online on
--train-frames plain ticks (untimed); then, from the same settled snapshot,
--steps ticks are timed with the plain warm start and --steps with the
learned one, each as CUDA-graph replays of two ticks. `value` is the learned
arm's steps/s with the state resident in HBM, timed with CUDA events on the
world's stream (max over ranks); the plain
arm's steps/s and both arms' sweep counts are in `config`. `e2e` is the
learned arm through the C ABI with host buffers (state upload from pinned
host memory, tick, state download each step). Multi-GPU runs independent replicas
(the coupled pile does not shard). Reference arm (--impl reference): the CPU
restatement of the reference's serial Slang CPU driver (oracle/, one core),
on the same state and schedule, over a bounded number of ticks: the oracle
first steps the same --warmup ticks as the GPU arms (untimed, so its contact
cache is as warm as theirs), then times --cpu-ticks ticks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "parallel-mater_b200"))

METRIC = "steps/sec at 64k boxes to equal residual: learned warm-start vs plain GPU AVBD"
GRID = (64, 32, 32)
SEED = 4
SETTLED = os.path.join(ROOT, "tests", "golden", "settled_pile_64x32x32.npz")
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "k_solve_pile65k.md")
NORMS = {"max": 0, "rms": 1, "p999": 2}
LANE_POLICIES = ["8/16/32 by colour size", "8", "8/16/32 by body rows, heaviest first",
                 "8/16/32 by colour size, bodies claimed dynamically",
                 "a body per thread in large colours, else 8/16/32 by colour size"]
SOLVE_THREADS = [512, 384, 256, 512, 384]  # plans 3, 4: the staged solve with fused duals


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pmb", choices=["pmb", "reference"])
    ap.add_argument("--tolerance", type=float, default=1e-4)
    ap.add_argument("--max-iterations", type=int, default=64)
    ap.add_argument("--residual-norm", default="p999", choices=["p999", "max", "rms"],
                    help="residual the schedule tests: 99.9th percentile of the row violations (default), "
                         "largest row violation, or RMS over the rows")
    ap.add_argument("--cpu-ticks", type=int, default=1, help="ticks timed by the CPU baseline leg")
    ap.add_argument("--contact-capacity", type=int, default=0,
                    help="contact-point capacity of the world (0: the library default, 64 per body)")
    ap.add_argument("--train-frames", type=int, default=200, help="plain ticks of online MLP training")
    ap.add_argument("--mlp-lr", type=float, default=3e-3)
    ap.add_argument("--mlp-steps", type=int, default=4, help="Adam steps per training frame")
    ap.add_argument("--workload", default="pile65k", choices=["pile65k", "batched"],
                    help="pile65k: the 65,536-box pile (default); batched: 1,024 independent scenes")
    ap.add_argument("--scenes", type=int, default=1024, help="batched: scene count")
    ap.add_argument("--settle", type=int, default=120, help="batched: plain ticks from the spawn before timing")
    ap.add_argument("--cpu-scenes", type=int, default=48, help="batched: scenes in the CPU baseline sample")
    ap.add_argument("--plan", default="", help="solve launch plan 'variant,policy' instead of the autotuner's")
    return ap.parse_args()


def choose_plan(world, desc, args):
    """The launch plan: --plan if given (set at once), else the autotuner's
    pick on this workload (state restored afterwards)."""
    if args.plan:
        v, p = (int(x) for x in args.plan.split(","))
        world.set_launch_plan(v, p)
        return v, p
    v, p, _ = world.autotune(desc, ticks=6)  # plans 5 % apart need more than a few ticks to tell apart
    return v, p


def load_scene():
    from pmb200 import scenes
    scene = scenes.box_pile(GRID, seed=SEED)
    z = np.load(SETTLED)
    scene.states = z["states"].astype(np.float32).view(scenes.STATE_DTYPE).reshape(-1).copy()
    return scene


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def solve_bytes(stats, n_dynamic):
    """Algorithmic bytes of the solve kernel for one tick (per iteration:
    primal 124 B per body + 2 x 112 B per contact point, dual 160 B per
    contact point), over both phases when the impact phase ran."""
    per_iter = 124 * n_dynamic + 384 * int(stats["contacts"])
    phases = 2 if int(stats["impact"]) else 1
    return phases * int(stats["iterations"]) * per_iter


def cpu_baseline(scene, desc, ticks, warm=0):
    """Steps/s of the CPU oracle over `ticks` ticks, after `warm` untimed
    ticks with the same schedule (the GPU arms' warm-up, so the contact cache
    and warm starts are as warm as theirs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    w = O.OracleWorld(scene)
    for _ in range(warm):
        w.step(desc)
    t0 = time.perf_counter()
    stats = None
    for _ in range(ticks):
        stats = w.step(desc)
    dt = time.perf_counter() - t0
    return ticks / dt, stats


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = load_scene()
    desc = scene.step_desc(residual_tolerance=args.tolerance, max_iterations=args.max_iterations,
                           residual_norm=NORMS[args.residual_norm])
    ticks = max(1, min(args.steps, args.cpu_ticks))
    value, stats = cpu_baseline(scene, desc, ticks, warm=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": ticks, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "box pile 64x32x32 (65,536 boxes), settled state, residual-driven AVBD",
                   "bodies": scene.n, "tolerance": args.tolerance, "residual_norm": args.residual_norm,
                   "max_iterations": args.max_iterations,
                   "iterations": int(stats["iterations"]), "contacts": int(stats["contacts"]),
                   "residual_row_max": float(stats["residual_max"])},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "port",
                         "sample": f"{ticks} warm tick(s) of the settled 65,541-body pile after {args.warmup} "
                                   f"untimed ones, {int(stats['iterations'])} sweeps; CPU restatement of the "
                                   "reference's serial Slang CPU driver (the generated driver needs slangc, absent)"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def graph_ticks(world, desc, steps, stream, torch, core, before=None):
    """CUDA-event time (ms) of `steps` ticks (even) as CUDA-graph replays of
    two ticks on the world's stream, from the world's snapshot, and the
    kernels they launch. The graph is captured and replayed once untimed
    first; `before` runs right before the timed replays."""
    world.restore()
    l0 = core.kernel_launches()
    world.capture(steps=2, desc=desc)
    per_replay = core.kernel_launches() - l0
    world.replay()
    world.restore()
    if before:
        before()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps // 2):
        world.replay()
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end), per_replay * (steps // 2)


def replay_stats(world, desc, steps):
    world.restore()
    return [world.step(desc) for _ in range(steps)]


def gpu_arm(args):
    import torch
    import torch.distributed as dist
    from pmb200 import core, scenes

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world_size > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    scene = load_scene()
    n_dyn = int((scene.bodies["motion"] == scenes.DYNAMIC).sum())
    norm = NORMS[args.residual_norm]
    plain = scene.step_desc(residual_tolerance=args.tolerance, max_iterations=args.max_iterations,
                            residual_norm=norm)
    learned = scene.step_desc(residual_tolerance=args.tolerance, max_iterations=args.max_iterations, warm_start=1,
                              residual_norm=norm)
    world = core.World(scene, device=local, contact_capacity=args.contact_capacity)
    stream = torch.cuda.Stream()             # a capturable (non-default) stream for the graph
    world.set_stream(stream.cuda_stream)
    steps = args.steps + (args.steps & 1)
    if args.plan:
        choose_plan(world, plain, args)

    def barrier():
        if world_size > 1:
            dist.barrier()

    def max_over_ranks(x):
        t = torch.tensor([x], device="cuda")
        if world_size > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        world.step(plain, stats=False)
    # The solve launch plan for this workload (autotuned unless --plan).
    plan_v, plan_p = choose_plan(world, plain, args)
    world.snapshot()

    # ---- online training of the warm-start MLP on plain ticks (untimed)
    t0 = time.perf_counter()
    world.mlp_attach(seed=1)
    world.mlp_train(True, lr=args.mlp_lr, steps_per_tick=args.mlp_steps)
    for _ in range(args.train_frames):
        world.step(plain, stats=False)
    _, mlp_loss, mlp_plain_loss, mlp_gate = world.mlp_params()
    world.mlp_train(False)
    train_s = time.perf_counter() - t0

    # ---- plain arm, device-resident, from the settled snapshot, as CUDA-graph
    # replays (clocks are sampled over both timed arms)
    sync = lambda: (barrier(), torch.cuda.synchronize())
    sampler = ClockSampler(local)
    sampler.start()
    plain_ms, _ = graph_ticks(world, plain, steps, stream, torch, core, before=sync)
    plain_ms = max_over_ranks(plain_ms)

    # ---- learned arm: the headline number
    torch.cuda.nvtx.range_push("learned_arm")
    learned_ms, launches = graph_ticks(world, learned, steps, stream, torch, core, before=sync)
    torch.cuda.nvtx.range_pop()
    learned_ms = max_over_ranks(learned_ms)
    barrier()
    clocks = sampler.stop()
    # per-tick statistics and the solve kernel's event time (plain launches)
    world.restore()
    world.solve_timer(True)
    torch.cuda.nvtx.range_push("learned_stats")
    learned_stats = [world.step(learned) for _ in range(steps)]
    torch.cuda.nvtx.range_pop()
    solve_ms, solve_launches = world.solve_timer(False)
    plain_stats = replay_stats(world, plain, steps)
    value = world_size * steps / (learned_ms * 1e-3)
    plain_value = world_size * steps / (plain_ms * 1e-3)

    alg_bytes = sum(solve_bytes(st, n_dyn) for st in learned_stats)
    achieved = alg_bytes / (solve_ms * 1e-3) / 1e9 if solve_ms > 0 else None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    # DRAM bytes per k_solve launch: the committed ncu capture of this
    # workload gives dram__bytes_read.sum + dram__bytes_write.sum per sweep
    # (one captured launch divided by its sweeps); scaled here by the mean
    # sweeps of this run's launches, since the schedule sets the sweep count.
    traffic = None
    try:
        with open(PROFILE_SUMMARY) as f:
            for line in f:
                if line.startswith("dram_bytes_per_sweep:"):
                    sweeps = sum((2 if int(st["impact"]) else 1) * int(st["iterations"]) for st in learned_stats)
                    traffic = float(line.split(":")[1]) * sweeps / max(1, solve_launches)
    except (OSError, ValueError):
        pass

    # ---- end to end through the C ABI with host buffers (learned arm)
    world.restore()
    host = torch.empty((scene.n, 13), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy().view(scenes.STATE_DTYPE).reshape(-1)
    host_np[:] = world.states()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        world.set_states(host_np)            # h2d: the step's input states
        world.step(learned, stats=False)
        world.states(out=host_np)            # d2h: the step's result
    torch.cuda.synchronize()
    e2e_value = world_size * steps / max_over_ranks(time.perf_counter() - t0)
    state_bytes = scene.n * 52

    cpu = None
    if rank == 0 and world_size == 1 and args.cpu_ticks > 0:
        cv, cst = cpu_baseline(scene, plain, args.cpu_ticks, warm=args.warmup)
        cpu = {"value": cv, "unit": "steps/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_ticks} warm tick(s) of the same settled pile after the GPU arms' "
                         f"{args.warmup} warm-up ticks (untimed), same schedule, plain warm start; serial CPU "
                         f"restatement (oracle/), {int(cst['iterations'])} sweeps, row-max residual "
                         f"{float(cst['residual_max']):.3g} m"}

    def mean(stats, key):
        return float(np.mean([int(st[key]) for st in stats]))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world_size,
            "steps": steps, "warmup": args.warmup, "ms_per_step": learned_ms / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "box pile 64x32x32 (65,536 boxes + ground and walls), settled state, "
                                   "legacy AVBD profile, residual-driven schedule; learned warm start "
                                   "(BF16 tcgen05 MLP, normal-row lambda and penalty prediction) vs plain",
                       "bodies": scene.n, "tolerance": args.tolerance, "residual_norm": args.residual_norm,
                       "max_iterations": args.max_iterations,
                       "plain_steps_per_s": plain_value, "learned_over_plain": value / plain_value,
                       "iterations_mean_learned": mean(learned_stats, "iterations"),
                       "iterations_mean_plain": mean(plain_stats, "iterations"),
                       "residual_row_max_learned": max(float(st["residual_max"]) for st in learned_stats),
                       "residual_row_max_plain": max(float(st["residual_max"]) for st in plain_stats),
                       "residual_rms_max_over_ticks_learned": max(float(st["residual"]) for st in learned_stats),
                       "residual_rms_max_over_ticks_plain": max(float(st["residual"]) for st in plain_stats),
                       "rows_over_tolerance_max_fraction_learned": max(float(st["residual_over"])
                                                                       for st in learned_stats),
                       "rows_over_tolerance_max_fraction_plain": max(float(st["residual_over"])
                                                                     for st in plain_stats),
                       "ticks_at_sweep_cap_learned": sum(int(st["iterations"]) >= args.max_iterations
                                                         for st in learned_stats),
                       "ticks_at_sweep_cap_plain": sum(int(st["iterations"]) >= args.max_iterations
                                                       for st in plain_stats),
                       "contacts_mean": mean(learned_stats, "contacts"),
                       "mlp_training": {"frames": args.train_frames, "adam_lr": args.mlp_lr,
                                        "steps_per_frame": args.mlp_steps, "seconds": round(train_s, 2),
                                        "applied": "normal-row lambda and penalty (apply mode 3)",
                                        "loss_over_plain_loss": mlp_loss / mlp_plain_loss if mlp_plain_loss else None,
                                        "gate_open": bool(mlp_gate)},
                       "launch_plan": {"solve_threads": SOLVE_THREADS[plan_v], "staged": plan_v >= 3,
                                       "lanes_per_body": LANE_POLICIES[plan_p]},
                       "parallelism": f"replicas x{world_size}",
                       "tick": "CUDA graph replays (one graph = two ticks); e2e: one pmb_world_step per tick",
                       "l2": "inputs larger than L2: per-tick working set ~%d MB (126 MB L2)" % int(
                           (mean(learned_stats, "contacts") * (8 + 9) * 16 + scene.n * 400 + 1.2e6 * 24) / 1e6)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "k_solve", "launches": solve_launches,
                         "kernel_ms_per_launch": solve_ms / max(1, solve_launches),
                         "peak_source": peak_src},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    world.close()
    if world_size > 1:
        dist.destroy_process_group()


BATCH_METRIC = "scene-steps/sec, 1,024 independent scenes (log-uniform 16-2048 bodies, piles and chains) per CUDA-graph tick"
BATCH_SEED = 5
BATCH_PROFILE = os.path.join(ROOT, "profiles", "k_solve_batch1024.md")


def batch_cpu_sample(count, ids):
    """CPU restatement (oracle/, one core) stepping each sampled scene on its
    own for one tick from the spawn; a batched world evolves every scene
    exactly as that scene stepped alone, so this is the same work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from pmb200 import scenes
    sizes, kinds = scenes.batched_plan(count, BATCH_SEED)
    parts = [scenes.batched_part(k, sizes[k], kinds[k], BATCH_SEED) for k in ids]
    bodies = sum(p.n for p in parts)
    elapsed = 0.0
    for p in parts:
        w = O.OracleWorld(p)
        t0 = time.perf_counter()
        w.step(p.step_desc())
        elapsed += time.perf_counter() - t0
    return len(parts) / elapsed, bodies


def batch_cpu_ids(count, want):
    """A bounded CPU sample: every (count // want)-th scene."""
    stride = max(1, count // max(1, want))
    return list(range(0, count, stride))[:want]


def reference_batched(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ids = batch_cpu_ids(args.scenes, args.cpu_scenes)
    value, bodies = batch_cpu_sample(args.scenes, ids)
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": value, "unit": "scene-steps/s",
        "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * args.scenes / value,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.scenes} independent scenes (config-5 mix, seed {BATCH_SEED}), first tick "
                               "from the spawn, per-scene iterations (piles 10, chains 20)"},
        "cpu_baseline": {"value": value, "unit": "scene-steps/s", "cores": 1, "kind": "port",
                         "sample": f"{len(ids)} of {args.scenes} scenes ({bodies} bodies), one tick each, stepped "
                                   "alone by the CPU restatement of the reference's serial Slang CPU driver"},
        "e2e": {"value": value, "unit": "scene-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def gpu_batched(args):
    """Config 5: the scenes are bin-packed over the ranks by body count; each
    rank steps its shard as one batched world, one CUDA-graph replay per two
    ticks, after settling from the spawn with the warm-start MLP trained
    online on the last --train-frames settling ticks. Arms: plain and learned
    warm start at the scenes' fixed iteration counts, from one snapshot."""
    import torch
    import torch.distributed as dist
    from pmb200 import core, scenes, shard

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world_size > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sizes, kinds = scenes.batched_plan(args.scenes, BATCH_SEED)
    mine = scenes.shard_scenes(sizes, world_size)[rank]
    scene = scenes.batched_scenes(args.scenes, BATCH_SEED, subset=mine)
    n_scenes = len(mine)
    dyn = scene.bodies["motion"] == scenes.DYNAMIC
    n_dyn = np.bincount(scene.body_scene[dyn], minlength=n_scenes)
    plain = scene.step_desc()
    learned = scene.step_desc(warm_start=1)
    world = core.World(scene, device=local, contact_capacity=args.contact_capacity)
    stream = torch.cuda.Stream()             # a capturable (non-default) stream for the graph
    world.set_stream(stream.cuda_stream)
    steps = args.steps + (args.steps & 1)
    if args.plan:
        choose_plan(world, plain, args)

    def barrier():
        if world_size > 1:
            dist.barrier()

    def max_over_ranks(x):
        t = torch.tensor([x], device="cuda")
        if world_size > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- settle from the spawn; MLP trained online on the last frames (untimed)
    t0 = time.perf_counter()
    train = min(args.train_frames, args.settle)
    for _ in range(args.settle - train):
        world.step(plain, stats=False)
    world.mlp_attach(seed=1)
    # Fixed per-scene sweep budgets: the learned warm start changes only the
    # residual here, and the penalty-only prediction keeps more scenes at or
    # below the plain residual than the lambda-and-penalty default.
    world.mlp_apply_mode(2)
    world.mlp_train(True, lr=args.mlp_lr, steps_per_tick=args.mlp_steps)
    for _ in range(train):
        world.step(plain, stats=False)
    _, mlp_loss, mlp_plain_loss, mlp_gate = world.mlp_params()
    world.mlp_train(False)
    for _ in range(args.warmup):
        world.step(plain, stats=False)
    status = int(world.step(plain)["status"])
    if status:
        raise RuntimeError("batched world status: %s" % core.status_names(status))
    settle_s = time.perf_counter() - t0
    plan_v, plan_p = choose_plan(world, plain, args)
    world.snapshot()

    def graph_arm(desc):
        world.restore()
        l0 = core.kernel_launches()
        world.capture(steps=2, desc=desc)
        per_replay = core.kernel_launches() - l0
        world.restore()
        world.replay()                       # untimed: first replay uploads the graph
        world.restore()
        barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps // 2):
            world.replay()
        end.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(start.elapsed_time(end)), per_replay * (steps // 2)

    plain_ms, _ = graph_arm(plain)
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.nvtx.range_push("learned_arm")
    learned_ms, launches = graph_arm(learned)
    torch.cuda.nvtx.range_pop()
    barrier()
    clocks = sampler.stop()

    def scene_trace(desc, timer=False):
        """Per tick and scene: residual RMS, residual max, sweeps, contacts."""
        world.restore()
        if timer:
            world.solve_timer(True)
        rms, mx, its, cts = [], [], [], []
        for _ in range(steps):
            st = world.step(desc)
            if int(st["status"]):
                raise RuntimeError("batched world status: %s" % core.status_names(int(st["status"])))
            r, m, i, c = world.scene_stats()
            rms.append(r), mx.append(m), its.append(i), cts.append(c)
        solve = world.solve_timer(False) if timer else (0.0, 0)
        return np.array(rms), np.array(mx), np.array(its), np.array(cts), solve

    p_rms, p_mx, p_its, p_cts, _ = scene_trace(plain)
    l_rms, l_mx, l_its, l_cts, (solve_ms, solve_launches) = scene_trace(learned, timer=True)
    # phase-0 algorithmic bytes of k_solve (per sweep: 124 B per dynamic body,
    # 384 B per contact point), summed over scenes and ticks
    alg_bytes = float(np.sum(l_its * (124.0 * n_dyn[None, :] + 384.0 * l_cts)))
    achieved = alg_bytes / (solve_ms * 1e-3) / 1e9 if solve_ms > 0 else None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    traffic = None
    try:
        with open(BATCH_PROFILE) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    traffic = float(line.split(":")[1])
    except (OSError, ValueError):
        pass

    # ---- end to end through the C ABI with host buffers (learned arm)
    world.restore()
    host = torch.empty((scene.n, 13), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy().view(scenes.STATE_DTYPE).reshape(-1)
    host_np[:] = world.states()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        world.set_states(host_np)
        world.step(learned, stats=False)
        world.states(out=host_np)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)

    # per-scene metrics of every rank, in global scene order
    per_scene = np.stack([p_rms.mean(0), l_rms.mean(0), p_mx.max(0), l_mx.max(0),
                          p_its.mean(0), l_cts.mean(0), n_dyn], axis=1).astype(np.float64)
    allm = shard.gather_by_scene(mine, per_scene, args.scenes, world_size)
    bodies_all = shard.gather_by_scene(mine, np.bincount(scene.body_scene, minlength=n_scenes), args.scenes,
                                       world_size)
    total_bodies = int(bodies_all.sum())
    cpu = None
    if rank == 0 and world_size == 1 and args.cpu_scenes > 0:
        ids = batch_cpu_ids(args.scenes, args.cpu_scenes)
        cv, cb = batch_cpu_sample(args.scenes, ids)
        cpu = {"value": cv, "unit": "scene-steps/s", "cores": 1, "kind": "port",
               "sample": f"{len(ids)} of {args.scenes} scenes ({cb} bodies), first tick from the spawn, each "
                         "stepped alone by the serial CPU restatement (oracle/)"}
    if rank == 0:
        value = args.scenes * steps / (learned_ms * 1e-3)
        plain_value = args.scenes * steps / (plain_ms * 1e-3)
        sweeps = float(np.sum(allm[:, 4] * allm[:, 6]))       # sweeps x dynamic bodies, per tick
        ratio = allm[:, 1] / np.maximum(allm[:, 0], 1e-30)
        has = allm[:, 0] > 0
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": "scene-steps/s", "n_gpus": world_size,
            "steps": steps, "warmup": args.warmup, "ms_per_step": learned_ms / steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"{args.scenes} independent scenes, body counts log-uniform [16,2048], "
                                   "box piles (10 sweeps) and joint chains (20 sweeps) 50/50, seed 5; legacy "
                                   f"profile; {args.settle} settling ticks from the spawn, then timed",
                       "bodies": total_bodies, "scenes_per_rank": n_scenes,
                       "tick": "one CUDA graph replay per 2 ticks",
                       "body_updates_per_s": sweeps * value / args.scenes,
                       "plain_scene_steps_per_s": plain_value, "learned_over_plain": value / plain_value,
                       "residual_rms_median_plain": float(np.median(allm[has, 0])) if has.any() else None,
                       "residual_rms_median_learned": float(np.median(allm[has, 1])) if has.any() else None,
                       "residual_max_plain": float(allm[:, 2].max()),
                       "residual_max_learned": float(allm[:, 3].max()),
                       "scenes_learned_at_or_below_plain": int(np.sum(ratio[has] <= 1.0)),
                       "scenes_learned_above_10x_plain": int(np.sum(allm[has, 3] > 10.0 * np.maximum(allm[has, 2], 1e-6))),
                       "scenes_with_contacts": int(has.sum()),
                       "mlp_training": {"frames": train, "adam_lr": args.mlp_lr, "steps_per_frame": args.mlp_steps,
                                        "loss_over_plain_loss": mlp_loss / mlp_plain_loss if mlp_plain_loss else None,
                                        "gate_open": bool(mlp_gate), "applied": "normal-row penalty (apply mode 2)"},
                       "settle_seconds": round(settle_s, 1),
                       "launch_plan": {"solve_threads": SOLVE_THREADS[plan_v], "staged": plan_v >= 3,
                                       "lanes_per_body": LANE_POLICIES[plan_p]},
                       "parallelism": f"scenes bin-packed by body count over {world_size} GPU(s)",
                       "l2": "inputs larger than L2 (per-tick working set several hundred MB)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "k_solve", "launches": solve_launches,
                         "kernel_ms_per_launch": solve_ms / max(1, solve_launches),
                         "bytes": "phase-0 sweeps only (impact-phase sweeps timed but not counted)",
                         "peak_source": peak_src},
            "cpu_baseline": cpu,
            "e2e": {"value": args.scenes * steps / e2e_s, "unit": "scene-steps/s",
                    "h2d_bytes_per_step": total_bodies * 52, "d2h_bytes_per_step": total_bodies * 52},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    world.close()
    if world_size > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.workload == "batched":
        (reference_batched if args.impl == "reference" else gpu_batched)(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
