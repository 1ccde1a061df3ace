"""Benchmark: rigid body-steps/s of the Dynamis step on the 262,144-body mixed pile.

One step = World::step over the whole world (broadphase, sort, pairs, narrowphase, islands,
2 substeps of the contact solve, sleep), replayed as one CUDA graph. The workload is the seeded
mixed pile (50% boxes, 30% spheres, 20% hulls, ground plane) advanced by --setup untimed steps so
the timed steps run on a forming pile rather than on the free-falling lattice.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line. `value` is device-resident throughput (states stay in HBM); `e2e` is the
same metric through the public C ABI with the body states uploaded from and downloaded to pinned
host memory every step. The reference arm (--impl reference) times the CPU restatement of the
step (the reference itself is Rust/WGSL on wgpu and cannot run on this machine).
With N > 1 (torchrun) every rank steps its own replica of the world: the single-world step has no
natural shard, so scaling is weak (replicas only) and there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "rigid body-steps/s at 256K bodies; batched-worlds & adjoint step/s vs plain"
UNIT = "body-steps/s"
DT = 1.0 / 60.0
WORKLOAD_DT = {"hanging_chains_8192": 1.0 / 120.0, "hanging_chains_131072": 1.0 / 120.0}


def dt_of(workload: str) -> float:
    """The timestep the workload's scene is specified at (1/120 s for the joint chains)."""
    return WORKLOAD_DT.get(workload, DT)
_T0 = time.perf_counter()


def log(message: str) -> None:
    """Progress on stderr (the JSON result is the only stdout line)."""
    print(f"[bench {time.perf_counter() - _T0:8.1f}s] {message}", file=sys.stderr, flush=True)


def peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [p.strip() for p in out.stdout.strip().split(",")]
                if len(parts) == 6:
                    self.samples.append(parts)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# DRAM bytes the narrowphase stage moved per candidate pair, measured with ncu on the formed
# 32,768-body pile; the full-size workload is too large for a multi-metric capture, and the traffic
# grows with the pair count.
NARROWPHASE_DRAM_BYTES_PER_PAIR = 250.0


def stage_bytes(stage: str, m: dict, params: dict) -> float:
    """Algorithmic (compulsory) HBM bytes of one launch of a stage's kernel pair, from the counts
    of the same step: K colliders, E entries, P pairs, C contacts, R solver rows, L live bodies."""
    K, E, P, C, R_, L = m["K"], m["E"], m["P"], m["C"], m["R"], m["L"]
    J = m.get("J", 0)
    # a ball joint per sweep (two sweeps per pass): 112 B of descriptor, two 92 B bodies read and
    # their velocities (or poses) written back, 12 B of accumulated impulse
    joint = 2 * (112.0 + 2 * 92.0 + 2 * 24.0 + 12.0) * J
    if stage == "velocity":     # one Jacobi iteration: joints, solve over contacts + apply over rows
        return 472.0 * C + 72.0 * R_ + joint
    if stage == "position":     # one position iteration
        return 200.0 * C + 64.0 * R_ + joint
    if stage == "narrowphase":
        return 596.0 * P
    if stage == "aabb":
        return 164.0 * K
    if stage == "entries":
        return 40.0 * E
    if stage == "entry_sort":
        return 16.0 * E * 4
    if stage == "pairs":
        return 40.0 * E + 8.0 * P
    if stage == "compact":   # contact keys (12 B), their sort (2 x 12 B a pass), the 352 B gather
        return 12.0 * C + 24.0 * C * 2 * params["contact_words"] + 2 * 352.0 * C
    if stage == "integrate":
        return 152.0 * L
    if stage == "islands":   # link over contacts (two passes), flatten and aggregate over the rows
        return 44.0 * C + 20.0 * R_
    return 0.0


LAUNCHES = {"velocity": lambda p: p["substeps"] * p["solve_iterations"],
            "position": lambda p: p["substeps"] * p["position_iterations"],
            "integrate": lambda p: p["substeps"]}


# Pair slots reserved per collider (World(capacity=...), the reference's kept reservation,
# crates/dynamis-world/tests/suite/capacity.rs:228: a reservation serves a whole scene without a second
# allocation). The formed mixed pile asks for up to ~18 pairs per collider in the timed steps; the
# stream widens by itself past half of its size, so 48 keeps a widening (a wait for the queued steps,
# new buffers and a new step graph) out of the timed region. Smaller streams are covered by the tests.
PAIR_SLOTS_PER_COLLIDER = 48


def build_world(workload: str, device: int):
    from dynamis_b200 import World, scenes

    scene = scenes.WORKLOADS[workload]()
    world = World(device=device, capacity={"pairs": PAIR_SLOTS_PER_COLLIDER * (len(scene.colliders) + 1)})
    t0 = time.perf_counter()
    scene.build(world)
    return world, scene, time.perf_counter() - t0


def long_run_checks(world, dt: float, before: dict, top: float) -> dict:
    """The long-run bounds at the end of the setup steps: total energy not above its start, no
    body faster than free fall from the scene's top, the deepest contact overlap, the pile's mean
    velocity."""
    from dynamis_b200 import diagnostics

    after = diagnostics.summary(world, dt)
    speed = np.linalg.norm(world.read_states()["velocity"].astype(np.float64), axis=1)
    bound = float(np.sqrt(2.0 * 9.81 * max(top, 0.0)))
    faster = int((speed > bound).sum())
    e0, e1 = before["energy"]["total"], after["energy"]["total"]
    return {"energy_start": e0, "energy_after_setup": e1, "energy_ratio": e1 / e0 if e0 else None,
            "free_fall_speed_bound": bound, "bodies_faster_than_free_fall": faster, "max_speed": float(speed.max()),
            "deepest_penetration": after["deepest_penetration"], "mean_velocity": after["mean_velocity"],
            "within_bounds": bool(e1 <= e0 * (1.0 + 1e-6) and faster == 0 and np.all(np.isfinite(speed)))}


def query_benchmark(world, batch: int = 16384, repeats: int = 3, seed: int = 9) -> dict:
    """Scene queries on the world as it stands (the formed pile): a batch of rays cast down onto it
    from above the lattice and a batch of sphere overlaps inside it, each through dyn_query (which
    first rebuilds the grid index from the current states), timed on the host around the whole call,
    best of `repeats`."""
    from dynamis_b200 import records as R

    rng = np.random.default_rng(seed)
    s = world.read_states()["position"]
    lo, hi = s.min(axis=0), s.max(axis=0)
    origins = rng.uniform(lo, hi, size=(batch, 3)).astype(np.float32)
    rays = np.concatenate([R.ray_query((o[0], hi[1] + 5.0, o[2]), (0, -1, 0), float(hi[1] - lo[1] + 10.0),
                                       R.query_filter(max_hits=4)) for o in origins])
    spheres = np.concatenate([R.sphere_query(o, 0.75, R.query_filter(max_hits=8)) for o in origins])
    out = {"batch": batch}
    for name, records in (("rays", rays), ("spheres", spheres)):
        best = float("inf")
        hits = 0
        for _ in range(repeats):
            t0 = time.perf_counter()
            q, _ = world.query(records)
            best = min(best, time.perf_counter() - t0)
            hits = int(q["count"].sum())
        out[name] = {"ms": round(best * 1e3, 3), "queries_per_s": round(batch / best, 1), "hits": hits}
    return out


def resting_benchmark(device: int, side: int = 512, steps: int = 50) -> dict:
    """A resting world: the 262,144 boxes of scenes.resting_field stepped until every body sleeps,
    then `steps` steps timed with CUDA events on the world's stream, with the grid counters of the
    last one (a resting world emits and sorts no grid entry: its entries stay in the kept resting
    run)."""
    import torch

    from dynamis_b200 import World, records as R, scenes

    dt = 1.0 / 60.0
    world = World(device=device)
    scenes.resting_field(side).build(world)
    stream = torch.cuda.Stream(device=device)
    world.set_stream(stream.cuda_stream)
    slept = None
    for i in range(600):
        world.step(dt)
        if i % 20 == 19:
            world.wait()
            if world.measured()[R.COUNTER["ACTIVE"]] == 0:
                slept = i + 1
                break
    for _ in range(3):
        world.step(dt)
    world.wait()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        world.step(dt)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end) / steps
    m = world.measured()
    out = {"bodies": world.sizes()["bodies"], "asleep_after_steps": slept, "ms_per_step": round(ms, 4),
           "counters": {k: int(m[R.COUNTER[k]]) for k in ("ACTIVE", "ENTRIES", "RESTING_ENTRIES", "RESTING_REBUILD",
                                                          "IMMOVABLE_EMITTED", "PAIRS")}}
    world.close()
    log(f"resting field: {out}")
    return out


def guarded_run(args, dt: float, device: int) -> dict:
    """The same workload with the row-mass guard on (dyn_set_solver_guard): the same setup, warm-up
    and timed steps, its setup bounds, its device time per step."""
    import torch

    from dynamis_b200 import diagnostics
    from dynamis_b200 import records as R

    world, scene, _ = build_world(args.workload, device)
    world.set_solver_guard(R.SOLVER_GUARD_ROW_MASS)
    stream = torch.cuda.Stream(device=device)
    world.set_stream(stream.cuda_stream)
    before = diagnostics.summary(world, dt, stepped=False)
    top = float(world.read_states()["position"][:, 1].max())
    for _ in range(args.setup):
        world.step(dt)
    world.wait()
    checks = long_run_checks(world, dt, before, top)
    for _ in range(args.warmup):
        world.step(dt)
    world.wait()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        world.step(dt)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end) / args.steps
    bodies = world.sizes()["bodies"]
    world.close()
    log(f"guarded: {ms:.3f} ms/step; setup checks {checks}")
    return {"solver_guard": "row_mass", "ms_per_step": ms, "value": bodies / (ms * 1e-3), "unit": UNIT,
            "setup_checks": checks}


def run_ours(args, rank: int, world_size: int, local_rank: int):
    import torch

    from dynamis_b200 import diagnostics
    from dynamis_b200 import records as R

    torch.cuda.set_device(local_rank)
    DT = dt_of(args.workload)
    world, scene, build_s = build_world(args.workload, local_rank)
    bodies = world.sizes()["bodies"]
    log(f"scene {args.workload}: {bodies} bodies built in {build_s:.1f}s")
    stream = torch.cuda.Stream(device=local_rank)
    world.set_stream(stream.cuda_stream)
    before = diagnostics.summary(world, DT, stepped=False)
    top = float(world.read_states()["position"][:, 1].max())
    for i in range(args.setup):
        world.step(DT)
        if i % 20 == 19:
            world.wait()
            log(f"setup step {i + 1}/{args.setup}")
    world.wait()
    log("setup done")
    setup_checks = long_run_checks(world, DT, before, top)
    log(f"setup checks {setup_checks}")
    launch = {"tuned": False}
    if not args.no_tune:
        from dynamis_b200 import tuning

        t0 = time.perf_counter()
        shapes, tuned_ms, ran = tuning.tuned(world, args.workload, DT, args.tuning_cache)
        launch = {**shapes, "tuned": ran, "tuner_ms_per_step": tuned_ms, "tune_s": round(time.perf_counter() - t0, 2)}
        log(f"launch shapes {launch}")
    for _ in range(args.warmup):
        world.step(DT)
    world.wait()
    # the end-to-end run below starts again from this state (World::snapshot / restore), so both
    # numbers describe the same steps of a pile that keeps getting denser
    start_state = world.snapshot()
    dist = None
    if world_size > 1:
        import torch.distributed as dist
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            world.step(DT)
        end.record(stream)
        end.synchronize()
    world.wait()
    ms = start.elapsed_time(end)
    log(f"timed {args.steps} steps: {ms / args.steps:.3f} ms/step")
    log("counts " + str({k: int(world.measured()[R.COUNTER[k]]) for k in ("ENTRIES", "PAIRS", "CONTACTS", "LIVE")}))
    ms = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    if dist:
        dist.barrier()
    m = world.measured()
    counts = {"K": world.sizes()["colliders"], "E": int(m[R.COUNTER["ENTRIES"]] + m[R.COUNTER["RESTING_ENTRIES"]] + m[R.COUNTER["IMMOVABLE_ENTRIES"]]),
              "P": int(m[R.COUNTER["PAIRS"]]), "C": int(m[R.COUNTER["CONTACTS"]]), "R": int(m[R.COUNTER["SOLVER_ROWS"]]),
              "L": int(m[R.COUNTER["LIVE"]]), "J": world.constraint_count(),
              "refused_pairs": int(m[R.COUNTER["REFUSED_PAIRS"]]),
              "refused_contacts": int(m[R.COUNTER["REFUSED_CONTACTS"]]), "pair_stream": world.stream_capacity()["pairs"],
              "pair_stream_reserved": PAIR_SLOTS_PER_COLLIDER * (len(scene.colliders) + 1)}
    launches_per_step = world.step_kernel_count()
    # per-stage breakdown: one more step run eagerly with CUDA events between stages
    world.set_timing(True)
    world.step(DT)
    world.wait()
    stages = world.stage_timings()
    world.set_timing(False)
    log("stages " + ", ".join(f"{k}={v:.3f}" for k, v in stages.items()))
    params = {"substeps": int(world.config["substeps"][0]), "solve_iterations": int(world.config["solve_iterations"][0]),
              "position_iterations": int(world.config["position_iterations"][0]),
              "contact_words": int(np.ceil(np.ceil(np.log2(max(counts["K"] - 1, 1) + 1)) / 8)) or 1}
    dominant = max(stages, key=stages.get)
    launches = LAUNCHES.get(dominant, lambda p: 1)(params)
    per_launch_ms = stages[dominant] / launches
    algo = stage_bytes(dominant, counts, params)
    pk = peaks()
    achieved = algo / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    stage_frac = {}
    for stage, stage_ms in stages.items():
        moved = stage_bytes(stage, counts, params) * LAUNCHES.get(stage, lambda p: 1)(params)
        if moved > 0 and stage_ms > 0:
            stage_frac[stage] = round(moved / (stage_ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4)
    # end to end through the C ABI with pinned host buffers, over the same steps as `value`: the world
    # goes back to the post-warm-up snapshot; one untimed round trip first, then back again
    e2e_steps = args.steps
    host = torch.empty(bodies * R.BODY_STATE.itemsize, dtype=torch.uint8, pin_memory=True)
    host_out = torch.empty_like(host, pin_memory=True)
    states_in = host.numpy().view(R.BODY_STATE)
    states_out = host_out.numpy().view(R.BODY_STATE)
    from dynamis_b200._native import lib, ptr

    world.restore(start_state)
    states_in[:] = world.read_states()
    world.upload_states(states_in)
    world.step(DT)
    world._check(lib.dyn_download_states(world._h, ptr(states_out), bodies))
    world.restore(start_state)
    start_state.close()
    states_in[:] = world.read_states()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        world.upload_states(states_in)
        world.step(DT)
        world._check(lib.dyn_download_states(world._h, ptr(states_out), bodies))
        states_in, states_out = states_out, states_in  # the result feeds the next step
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local_rank}")
    log(f"e2e {e2e_steps} steps: {e2e_s / e2e_steps * 1e3:.3f} ms/step")
    result = {
        "metric": METRIC, "value": whole_job_rate(bodies * args.steps, world_size, ms * 1e-3), "unit": UNIT,
        "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "bodies": bodies, "setup_steps": args.setup, "dt": DT,
                   "parallelism": f"replicas{world_size}" if world_size > 1 else "single-world",
                   "l2": "working set > 126 MB L2 (no flush between steps)", "counts_last_step": counts,
                   "scene_build_s": round(build_s, 2)},
        "e2e": {"value": whole_job_rate(bodies * e2e_steps, world_size, e2e_s), "unit": UNIT, "h2d_bytes_per_step": bodies * R.BODY_STATE.itemsize,
                "d2h_bytes_per_step": bodies * R.BODY_STATE.itemsize},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"],
                     "traffic": NARROWPHASE_DRAM_BYTES_PER_PAIR * counts["P"] if dominant == "narrowphase" else None,
                     "peak_source": pk["source"],
                     "algorithmic_bytes_per_launch": algo, "ms_per_launch": per_launch_ms},
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "stage_frac": stage_frac,
        "launch_config": launch,
        "setup_checks": setup_checks,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks.summary(),
    }
    # the measurements beside the headline run at N = 1 only (the scaling runs time the replicas)
    extras = world_size == 1
    if extras and not args.no_queries:
        result["queries"] = query_benchmark(world)
        log(f"queries {result['queries']}")
    if extras and not args.no_resting:
        result["resting"] = resting_benchmark(local_rank)
    if extras and not args.no_batch:
        result["batch"] = batch_benchmark(args, local_rank)
    if extras and not args.no_guarded:
        result["guarded"] = guarded_run(args, DT, local_rank)
    if extras and not args.no_adjoint:
        result["adjoint"] = adjoint_benchmark(local_rank, steps=args.adjoint_steps, settle=args.adjoint_setup)
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(world, budget_s=args.cpu_budget, dt=DT)
    world.close()
    return result


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's value: a replicated job ends when its slowest replica does."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world_size: int, seconds: float) -> float:
    """Units all ranks processed per second of the slowest rank."""
    return units_per_rank * world_size / seconds


ADJOINT_WORKLOAD = "differentiable_towers_256"


def adjoint_benchmark(device: int, steps: int = 120, settle: int = 60, interval: int = 10) -> dict:
    """The differentiable workload: 256 tower worlds (8-high, 4 x 4 unit boxes each, masses drawn
    U(0.5, 2) kg, friction per world U(0.3, 0.8)) and a sphere per world launched at U(3, 8) m/s
    toward its tower, sleeping off, dt 1/120 s. Two identical worlds settle `settle` steps; then one
    steps `steps` times plainly (the plain forward) and the other records the same steps with
    checkpoints every `interval` steps and reverses all of them (dyn_backward, which replays each
    segment from its checkpoint, narrowphase included). Times are CUDA events on each world's stream."""
    import torch

    from dynamis_b200 import World, records as R, scenes

    dt = 1.0 / 120.0
    scene = scenes.WORKLOADS[ADJOINT_WORKLOAD]()
    worlds, streams = [], []
    for _ in range(2):
        w = World(device=device, sleep_time=float("inf"))
        scene.build(w)
        stream = torch.cuda.Stream(device=device)
        w.set_stream(stream.cuda_stream)
        for _ in range(settle):
            w.step(dt)
        w.wait()
        worlds.append(w)
        streams.append(stream)
    plain, taped = worlds
    bodies = plain.sizes()["bodies"]
    # warm-up: both worlds take the same `steps` steps; the taped one records them and reverses one,
    # so its tape, checkpoint blocks and reverse graph exist before the timed run (a tape of the same
    # shape allocates nothing), and the recorded end state is restored: the two stay identical
    for _ in range(steps):
        plain.step(dt)
    taped.tape_begin(interval)
    for _ in range(steps):
        taped.step(dt)
    taped.step_backward(np.zeros(bodies, R.BODY_GRAD), 1)
    taped.tape_end()
    for w in worlds:
        exported = w.export_scene()
        spheres = np.sort(exported["owners"][exported["colliders"]["kind"] == R.SHAPE_SPHERE]).astype(np.int64)
        states = w.read_states()
        states["velocity"][spheres] = scenes.sphere_launches(scene, states, spheres)
        w.upload_states(states)
    assert np.array_equal(plain.read_states()["position"], taped.read_states()["position"])

    def timed(stream, body):
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        body()
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end)

    def forward(w):
        for _ in range(steps):
            w.step(dt)

    forward_ms = timed(streams[0], lambda: forward(plain))
    taped.tape_begin(interval)
    taped_ms = timed(streams[1], lambda: forward(taped))
    final = taped.read_states()
    grad = np.zeros(bodies, R.BODY_GRAD)
    grad["position"] = 2.0 * final["position"]  # d/dx of the summed squared final positions
    holder = {}
    backward_ms = timed(streams[1], lambda: holder.update(out=taped.step_backward(grad, steps)))
    g = taped.param_grads()
    taped.tape_end()
    finite = bool(np.all(np.isfinite(holder["out"]["velocity"])) and np.all(np.isfinite(g["inverse_mass"])))
    for w in worlds:
        w.close()
    log(f"adjoint: plain forward {forward_ms:.1f} ms, taped forward {taped_ms:.1f} ms, backward {backward_ms:.1f} ms "
        f"for {steps} steps of {bodies} bodies")
    return {"workload": ADJOINT_WORKLOAD, "bodies": bodies, "steps": steps, "dt": dt, "checkpoint_interval": interval,
            "setup_steps": settle + steps, "forward_ms": forward_ms, "taped_forward_ms": taped_ms, "backward_ms": backward_ms,
            "fwd_bwd_over_fwd": (taped_ms + backward_ms) / forward_ms,
            "fwd_bwd_body_steps_per_s": bodies * steps / ((taped_ms + backward_ms) * 1e-3),
            "forward_body_steps_per_s": bodies * steps / (forward_ms * 1e-3), "gradients_finite": finite}


def batch_benchmark(args, device: int, worlds: int = 4096, setup: int = 5, warmup: int = 2, steps: int = 5) -> dict:
    """Batched worlds (the survey's fourth configuration): `worlds` sub-worlds in one World, one
    graph launch a step, against the same worlds as a loop of plain single-world steps (one World
    and one graph launch each, on one stream), every world of the loop timed, after the same setup
    and warm-up steps. Both sides are launch-bound for small worlds, so a short setup serves."""
    import torch

    from dynamis_b200 import World, scenes

    dt = DT
    parts = scenes.batched_world_parts(worlds)
    batch = World(device=device)
    scenes.batch(parts).build(batch)
    stream = torch.cuda.Stream(device=device)
    batch.set_stream(stream.cuda_stream)
    bodies = batch.sizes()["bodies"]
    for _ in range(setup + warmup):
        batch.step(dt)
    batch.wait()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        batch.step(dt)
    end.record(stream)
    end.synchronize()
    batch_ms = start.elapsed_time(end) / steps
    batch.close()
    loop = []
    for part in parts:
        w = World(device=device)
        part.build(w)
        w.set_stream(stream.cuda_stream)
        loop.append(w)
    for _ in range(setup + warmup):
        for w in loop:
            w.step(dt)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        for w in loop:
            w.step(dt)
    end.record(stream)
    end.synchronize()
    loop_ms = start.elapsed_time(end) / steps
    for w in loop:
        w.close()
    log(f"batch of {worlds} worlds ({bodies} bodies): {batch_ms:.2f} ms/step; loop of all {worlds}: {loop_ms:.1f} ms/step")
    return {"workload": f"batched_worlds_{worlds}", "worlds": worlds, "bodies": bodies, "setup_steps": setup,
            "steps": steps, "batch_ms_per_step": batch_ms, "batch_body_steps_per_s": bodies / (batch_ms * 1e-3),
            "loop": {"worlds": worlds, "ms_per_step": loop_ms, "timed": "every world, in full"},
            "speedup_vs_loop": loop_ms / batch_ms}


def cpu_baseline(world, budget_s: float = 20.0, dt: float = DT) -> dict:
    """The oracle (CPU restatement) stepping the same world state on every host thread, then one
    more step on a single thread."""
    from oracle import oracle as orc

    scene = world.export_scene()
    scene["states"] = world.read_states()
    oracle = orc.OracleWorld(scene, world.step_params(dt))
    cores = orc.threads()
    log(f"cpu baseline: oracle world built; {cores} threads")
    steps = 0
    t0 = time.perf_counter()
    while True:
        oracle.step(dt)
        steps += 1
        if time.perf_counter() - t0 > budget_s / 2 or steps >= 3:
            break
    elapsed = time.perf_counter() - t0
    n = len(scene["states"])
    single = None
    if budget_s > 0:
        orc.set_threads(1)
        t1 = time.perf_counter()
        oracle.step(dt)
        single = n / (time.perf_counter() - t1)
        orc.set_threads(cores)
    oracle.close()
    return {"value": n * steps / elapsed, "unit": UNIT, "cores": cores, "kind": "port",
            "single_thread_value": single,
            "sample": f"{steps} step(s) of the full {n}-body world from its current state on "
                      f"{cores} threads (OpenMP), then 1 step on one thread (single_thread_value)"}


def run_reference(args) -> dict:
    """The reference arm: the reference's step as the CPU restatement runs it (the reference itself is
    Rust + WGSL on wgpu and cannot run here), on every host thread. The arm uses no product code: the
    oracle builds the scene's records itself (oracle/scene.cpp restates the reference's spawn path and
    matches the library byte for byte), steps the same setup and warm-up steps, then times a bounded
    sample of steps, which it reports as its steps."""
    import os

    from dynamis_b200 import scenes
    from oracle import oracle as orc

    DT = dt_of(args.workload)
    scene = scenes.WORKLOADS[args.workload]()
    records = orc.scene_records(scene.bodies, scene.colliders, scene.hulls, scene.worlds, dt=DT)
    bodies = len(records["states"])
    world = orc.OracleWorld(records, records["params"])
    cores = orc.threads()
    t0 = time.perf_counter()
    for i in range(args.setup + args.warmup):
        world.step(DT)
        if i % 20 == 19:
            log(f"reference setup step {i + 1}/{args.setup + args.warmup}")
    log(f"reference setup: {args.setup + args.warmup} oracle steps in {time.perf_counter() - t0:.1f}s")
    budget = args.cpu_budget
    timed = 0
    t0 = time.perf_counter()
    while timed < max(1, min(args.steps, 3)):
        world.step(DT)
        timed += 1
        if time.perf_counter() - t0 > budget / 2:
            break
    elapsed = time.perf_counter() - t0
    world.close()
    value = bodies * timed / elapsed
    loaded = [line.split()[-1] for line in open(f"/proc/{os.getpid()}/maps") if line.rstrip().endswith(".so")]
    assert not any("libdynamis_cuda" in name for name in loaded), "the reference arm must not load the product"
    base = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{timed} step(s) of the full {bodies}-body world after {args.setup + args.warmup} setup and "
                      f"warm-up steps, all on the oracle (records built by the oracle), {cores} threads (OpenMP)"}
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": timed, "warmup": args.warmup, "ms_per_step": elapsed / timed * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "bodies": bodies, "setup_steps": args.setup, "dt": DT,
                       "parallelism": "single-world"},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--setup", type=int, default=120, help="untimed steps that form the pile before warm-up")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed_pile_262144")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-towers measurement")
    ap.add_argument("--no-guarded", action="store_true", help="skip the run with the row-mass guard")
    ap.add_argument("--no-queries", action="store_true", help="skip the scene-query measurement")
    ap.add_argument("--no-resting", action="store_true", help="skip the resting-world measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-worlds measurement")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuner)")
    ap.add_argument("--tuning-cache", default=None, help="JSON file of per-workload launch shapes to reuse and extend")
    ap.add_argument("--adjoint-only", action="store_true", help="print only the differentiable-towers measurement")
    ap.add_argument("--adjoint-steps", type=int, default=120)
    ap.add_argument("--adjoint-setup", type=int, default=60)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    if args.adjoint_only:
        import torch

        torch.cuda.set_device(local_rank)
        print(json.dumps(adjoint_benchmark(local_rank, steps=args.adjoint_steps, settle=args.adjoint_setup)))
        return
    if world_size > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    result = run_ours(args, rank, world_size, local_rank)
    if rank == 0:
        print(json.dumps(result))
    if world_size > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
