#!/usr/bin/env python
"""Benchmark of the per-step cloth pipeline (silk::World::solver_step).

Workload (N = 1): the 6.4K-vertex sheet of the benchmark's second
configuration -- an 80 x 80 grid (12,482 triangles, side 1 m, jitter
N(0, 1e-4) m from a fixed seed) on a static icosphere (subdivision 4, radius
0.3 m), self-collision and obstacle CCD on, float32, dt = 1/60, gravity
-9.81, CG relative tolerance fixed at 1e-5 -- in the contact regime: both arms
start from the CPU oracle's own state after 27 steps (24 of free fall, 3 in
contact; oracle/reference_state_c2_step27.npz, which also holds the MAS
partition both arms use), so they time the same steps (28, 29, ...) from the
same state.  A step is one solver_step.

Metric: steps/s (higher is better).  `value`: K steps timed with CUDA events
on the world's stream, inputs resident, a 256 MiB write flushing L2 before
each step (outside the events).  `e2e`: the same K steps again from the same
state through the public API with host buffers (obstacle position from
pinned memory + solver_step + cloth position into pinned memory, inside the
timed region).  The W warm-up steps run from the stored state before the
world is set back to it.

Multi-GPU: scenes are independent, so --gpus N runs N replicas (one process
per GPU, no collective on the data path; barrier + max over ranks only).

`--impl reference` times the CPU restatement of the reference algorithm
(oracle/; the reference itself cannot be built here) on all host cores from
the same stored state, as many of the same steps as fit the CPU budget.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOAD = "c2_sheet80_on_icosphere_r0.3_contact"
METRIC = "steps/s (6.4K-vertex sheet on sphere, active contact)"
C3_WORKLOAD = "c3_sheet316_on_icosphere_r0.6_first_contact"
STATE = ROOT / "oracle" / "reference_state_c2_step27.npz"
MODEL = ROOT / "silk_physics_b200" / "models" / "warm_start.npy"
TRAFFIC = ROOT / "profiles" / "cg_cluster_c2_contact.json"
SCENES = ROOT / "tests" / "golden" / "reference_scenes.npz"
C3_START_STEPS = 8  # free-fall steps before the drape's first contact step


def scene():
    from silk_physics_b200 import scenes as S

    return S.c2_scene()


def scene_c3():
    from silk_physics_b200 import scenes as S

    return S.c3_scene()


def stored_state():
    """(x, v, steps, perm, part_offsets) of the stored C2 contact state."""
    d = np.load(STATE)
    return (d["x"].reshape(-1), d["v"].reshape(-1), int(d["steps"]), d["perm"],
            d["part_offsets"])


def c3_start(V):
    """The drape's free-fall state right before its first contact step."""
    from silk_physics_b200 import scenes as S

    x, v = S.free_fall_state(V, C3_START_STEPS)
    return x.reshape(-1), v.reshape(-1)


def bench_config(args, V, F, SV, world_size: int) -> dict:
    """The workload description, identical in both arms."""
    return {"workload": WORKLOAD, "vertices": int(len(V)), "faces": int(len(F)),
            "obstacle_vertices": int(len(SV)),
            "start": "CPU oracle state after 27 steps (in contact), timed steps 28 on",
            "cg_rel_tol": args.cg_rel_tol if args.cg_rel_tol > 0 else "adaptive (reference)",
            "mas": "bf16" if args.bf16 else "fp32",
            "mas_partition": "host partition stored with the state",
            "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": f"replicas x{world_size}"}


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))



# Replicas plumbing (one process per GPU, no data-path collective): a process
# group with a short timeout, a barrier and the max over ranks of each rank's
# device time, and scenes sharded by rank.  The backend is "nccl" on GPUs and
# "gloo" in the CPU tests of this plumbing.
def dist_init(backend: str, timeout_s: int = 600) -> bool:
    """Start the process group when WORLD_SIZE > 1; True if one runs."""
    _, _, world_size = dist_env()
    if world_size <= 1:
        return False
    import torch.distributed as dist
    from datetime import timedelta

    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return True


def max_over_ranks(ms: float, device: str) -> float:
    """Largest value over the ranks (every rank takes part), then a barrier."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def shard(items, rank: int, world_size: int):
    """Items of this rank: every world_size-th, starting at its rank."""
    return items[rank::world_size]


def weak_value(units_per_rank_step: float, world_size: int, steps: int, ms: float) -> float:
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time."""
    return units_per_rank_step * world_size * steps / (ms / 1e3)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(f"/tmp/silk_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self) -> dict:
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines()]
        except Exception:
            rows = []
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}




def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_per_launch():
    """DRAM bytes per CG launch of a contact-regime solve, from the committed
    ncu summary (profiles/cg_cluster_c2_contact.json), or None."""
    if not TRAFFIC.exists():
        return None
    d = json.loads(TRAFFIC.read_text())
    return {"bytes": d["dram_bytes_per_launch"], "source": TRAFFIC.name,
            "captured": d.get("captured")}


def make_world(stream_handle, opts, V, F, SV, SF, model=False):
    from silk_physics_b200 import native as N

    w = N.World()
    r = w.init()
    if not r:
        raise RuntimeError(r.to_string())
    w.set_global_config(N.GlobalConfig(acceleration_z=-9.81))
    w.set_solver_options(opts)
    if stream_handle:
        w.set_stream(stream_handle)
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, [])
    assert r, r.to_string()
    r, hs = w.add_obstacle(N.CollisionConfig(), SV, SF)
    assert r, r.to_string()
    if model:
        from silk_physics_b200 import learned as L

        r = w.set_warm_start_model(L.load(str(MODEL)))
        assert r, r.to_string()
    return w, h, hs


def oracle_steps(x0, v0, perm, offs, V, F, SV, SF, cg_rel_tol, max_steps, budget_s):
    """The CPU restatement stepped from (x0, v0) on all host cores: per-step
    wall seconds of up to max_steps steps, stopping once budget_s is spent
    (at least one step), and their ADMM iterations."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    ow = pyoracle.OracleWorld(config=dict(acceleration=(0.0, 0.0, -9.81),
                                          fixed_linear_rel_tol=cg_rel_tol))
    h = ow.add_cloth(V, F, [], perm, offs)
    ow.add_obstacle(SV, SF)
    ow.set_state(h, x0, v0)
    times, admm = [], 0
    t0 = time.perf_counter()
    for _ in range(max_steps):
        a = time.perf_counter()
        assert ow.step() == 0
        times.append(time.perf_counter() - a)
        admm += ow.stats()["admm_iterations"]
        if time.perf_counter() - t0 > budget_s:
            break
    return times, admm


def replay_variant(N, torch, stream, flush, V, F, SV, SF, x0, v0, cg_rel_tol, bf16, learned,
                   extrap, reps):
    """Controlled A/B: `reps` times the same step from the same state (the
    world is set back to (x0, v0) before each), CUDA events around each
    step, L2 flushed before it."""
    opts = N.SolverOptions(fixed_linear_rel_tol=cg_rel_tol, profile=True, mas_bf16=bf16,
                           learned_warm_start=learned, admm_extrapolated_start=extrap)
    w, h, _ = make_world(stream.cuda_stream, opts, V, F, SV, SF, model=learned)
    assert w.set_cloth_state(h, x0, v0)
    assert w.solver_step()  # untimed: first-use setup of the world
    w.profile(reset=True)
    ms, keys = [], set()
    for k in range(reps):
        assert w.set_cloth_state(h, x0, v0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xff)
            a.record(stream)
        r = w.solver_step()
        b.record(stream)
        b.synchronize()
        assert r, r.to_string()
        ms.append(a.elapsed_time(b))
        s = w.step_stats()
        keys.add((s.admm_iterations, s.cg_iterations, s.contacts, s.outer_iterations))
    s = w.step_stats()
    prof = w.profile(reset=True)
    med = statistics.median(ms)
    return {"ms_per_step_median": round(med, 2), "ms_per_step": [round(t, 2) for t in ms],
            "value": round(1e3 / med, 4),
            "admm_iterations_per_step": s.admm_iterations,
            "outer_iterations": s.outer_iterations,
            "cg_iterations_per_step": s.cg_iterations,
            "cg_iterations_per_solve": round(s.cg_iterations / max(s.cg_solves, 1), 2),
            "first_solve_cg_iterations": s.cg_first_solve_iterations,
            "ms_per_admm_iteration": round(med / max(s.admm_iterations, 1), 4),
            "cg_kernel_ms_per_step": round(prof["cg_time_ms"] / reps, 2),
            "contact_gs_ms_per_step": round(prof["contact_gs_ms"] / reps, 2),
            "ccd_host_ms_per_step": round(prof["ccd_host_ms"] / reps, 2),
            "ccd_refit_host_ms_per_step": round(prof["ccd_refit_host_ms"] / reps, 2),
            "ccd_candidates_host_ms_per_step": round(prof["ccd_candidates_host_ms"] / reps, 2),
            "ccd_first_pass_ms_per_step": round(prof["ccd_first_pass_ms"] / reps, 2),
            "ccd_second_pass_ms_per_step": round(prof["ccd_second_pass_ms"] / reps, 2),
            "ccd_second_pass_queries_per_step": round(prof["ccd_second_pass_queries"] / reps, 1),
            "ccd_calls_per_step": round(prof["ccd_calls"] / reps, 1),
            "contacts": s.contacts, "replays_identical": len(keys) == 1,
            "learned_starts_taken": s.learned_starts,
            "extrapolated_starts_taken": s.extrapolated_starts}


def variants_ab(N, torch, stream, flush, args):
    """Plain FP32 MAS, BF16 MAS and the learned warm start, each replaying
    the same contact step from the same state: C2 from the stored oracle
    state, C3 from the drape's free-fall state before its first contact."""
    out = {}
    forms = (("plain_fp32", False, False, False), ("bf16", True, False, False),
             ("learned_bf16", True, True, False), ("extrapolated_fp32", False, False, True),
             ("learned_extrapolated_bf16", True, True, True))
    V, F, SV, SF = scene()
    x0, v0, s0, _, _ = stored_state()
    c2 = {"workload": WORKLOAD, "replayed_step": s0 + 1, "replays": args.variant_reps}
    for name, bf16, learned, extrap in forms:
        if learned and not MODEL.exists():
            continue
        c2[name] = replay_variant(N, torch, stream, flush, V, F, SV, SF, x0, v0,
                                  args.cg_rel_tol, bf16, learned, extrap, args.variant_reps)
    out["c2"] = c2
    V3, F3, SV3, SF3 = scene_c3()
    x3, v3 = c3_start(V3)
    c3 = {"workload": C3_WORKLOAD, "vertices": int(len(V3)), "faces": int(len(F3)),
          "replayed_step": C3_START_STEPS + 1, "replays": args.variant_reps}
    for name, bf16, learned, extrap in forms:
        if learned and not MODEL.exists():
            continue
        c3[name] = replay_variant(N, torch, stream, flush, V3, F3, SV3, SF3, x3, v3,
                                  args.cg_rel_tol, bf16, learned, extrap, args.variant_reps)
    for d in (c2, c3):
        for name in ("bf16", "learned_bf16", "extrapolated_fp32", "learned_extrapolated_bf16"):
            if name in d:
                d[name + "_over_plain"] = round(
                    d["plain_fp32"]["ms_per_step_median"] / d[name]["ms_per_step_median"], 3)
    out["c3"] = c3
    return out


def reference_scenes(N, steps_cloth_ball: int):
    """The reference's own example scenes (packaged in tests/golden/) through
    the headless driver with the reference's default solver settings
    (adaptive CG tolerance): dense_sheet.json (the README's 6K sheet, its 10
    steps) and cloth_ball.json (the same sheet on a ground plane and a
    sphere, first steps_cloth_ball steps).  Host wall time of solver_step."""
    from silk_physics_b200 import headless as H

    d = dict(np.load(SCENES))
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, steps in (("dense_sheet", None), ("cloth_ball", steps_cloth_ball)):
            text = bytes(d[f"{name}/json"]).decode()
            meshes = {o["mesh"]: (d[f"mesh/{o['mesh']}/verts"], d[f"mesh/{o['mesh']}/faces"])
                      for o in json.loads(text)["objects"]}
            path = H.write_scene(Path(tmp) / name, name, text, meshes)
            g = json.loads(text)["global"]
            _, wall = H.run(path, steps=steps, bench=True, log=None)
            # The first step of a fresh world also builds its solver layout
            # (partition, assembly, MAS plans); the rate is over the others.
            n = len(wall) - 1
            rest = sum(wall[1:])
            out[name] = {"steps_timed": n, "dt": g["dt"], "value": round(n / (rest / 1e3), 3),
                         "unit": "steps/s", "ms_per_step": round(rest / n, 2),
                         "first_step_ms_with_setup": round(wall[0], 1),
                         "max_inner_iteration": g["max_inner_iteration"],
                         "cg_tolerance": "adaptive (reference default)"}
    out["note"] = ("README.md:7 of the reference: 'maintain 40 FPS' on a 6K cloth mesh with "
                   "active collision, hardware, backend and settings unstated")
    return out


def config1(N, torch, stream, cg_rel_tol, steps, cpu_budget_s):
    """Config 1 as stated: the 32x32 sheet (two top corners pinned, default
    cloth and collision settings, self-collision on, no obstacle), 10 ADMM
    iterations per step, `steps` steps on the GPU timed with CUDA events
    (the first, which builds the solver layout, untimed), and the CPU
    restatement on all host cores for as many of the same steps as fit
    cpu_budget_s (None: skipped)."""
    from silk_physics_b200 import scenes as S

    V, F = S.grid_sheet(32, jitter=0.0, seed=7)
    P = S.top_corner_pins(32)
    w = N.World()
    assert w.init()
    w.set_stream(stream.cuda_stream)
    assert w.set_global_config(N.GlobalConfig(max_inner_iteration=10, admm_abs_tol=0.0,
                                              admm_rel_tol=0.0))
    assert w.set_solver_options(N.SolverOptions(fixed_linear_rel_tol=cg_rel_tol))
    r, h = w.add_cloth(N.ClothConfig(), N.CollisionConfig(), V, F, P)
    assert r, r.to_string()
    perm, offs = w.cloth_partition(h, len(V))
    assert w.solver_step()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    contacts = 0
    with torch.cuda.stream(stream):
        a.record(stream)
        for _ in range(steps - 1):
            assert w.solver_step()
            contacts = max(contacts, w.step_stats().contacts)
        b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / (steps - 1)
    out = {"workload": "c1_sheet32_pinned_selfcollision", "vertices": int(len(V)),
           "steps_timed": steps - 1, "value": round(1e3 / ms, 2), "unit": "steps/s",
           "ms_per_step": round(ms, 3), "admm_iterations_per_step": 10,
           "max_contacts": contacts, "cg_rel_tol": cg_rel_tol}
    if cpu_budget_s is not None:
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyoracle

        ow = pyoracle.OracleWorld(config=dict(max_inner_iteration=10, admm_abs_tol=0.0,
                                              admm_rel_tol=0.0, fixed_linear_rel_tol=cg_rel_tol))
        ow.add_cloth(V, F, P, perm, offs)
        t0 = time.perf_counter()
        n = 0
        while n < steps and (n == 0 or time.perf_counter() - t0 < cpu_budget_s):
            assert ow.step() == 0
            n += 1
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(n / sec, 4), "unit": "steps/s",
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"the first {n} of the same steps ({sec:.1f} s wall)"}
    return out


def run_ours(args) -> None:
    import torch

    rank, local_rank, world_size = dist_env()
    torch.cuda.set_device(local_rank)
    dist_init("nccl")
    from silk_physics_b200 import native as N

    V, F, SV, SF = scene()
    x0, v0, s0, perm_s, offs_s = stored_state()
    stream = torch.cuda.Stream()
    opts = N.SolverOptions(fixed_linear_rel_tol=args.cg_rel_tol, profile=True,
                           mas_bf16=args.bf16)
    w, h, hs = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    perm, offs = w.cloth_partition(h, len(V))
    assert np.array_equal(perm, perm_s) and np.array_equal(offs, offs_s), \
        "the stored state's partition is not the one this build computes"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    assert w.set_cloth_state(h, x0, v0)
    for _ in range(args.warmup):
        r = w.solver_step()
        assert r, r.to_string()
    assert w.set_cloth_state(h, x0, v0)
    w.profile(reset=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = admm = cg = solves = contacts = cluster_solves = 0
    per_step_admm = []
    if world_size > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xff)
                ev[k][0].record(stream)
            r = w.solver_step()
            ev[k][1].record(stream)
            assert r, r.to_string()
            st = w.step_stats()
            launches += st.kernel_launches
            admm += st.admm_iterations
            per_step_admm.append(st.admm_iterations)
            cg += st.cg_iterations
            solves += st.cg_solves
            cluster_solves += st.cg_cluster_solves
            contacts = st.contacts
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    prof = w.profile(reset=True)
    total_ms = max_over_ranks(total_ms, "cuda")
    value = weak_value(1, world_size, args.steps, total_ms)

    # End to end through the public API with host buffers, the same K steps
    # from the same state.
    assert w.set_cloth_state(h, x0, v0)
    pin_obs = torch.from_numpy(SV.ravel().copy()).pin_memory().numpy()
    pin_out = torch.empty(V.size, dtype=torch.float32).pin_memory().numpy()
    e2e_ms, e2e_admm = [], []
    w.profile(reset=True)
    torch.cuda.synchronize()
    for k in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xff)
        a.record(stream)
        w.set_obstacle_position(hs, pin_obs)
        r = w.solver_step()
        w.get_cloth_position(h, pin_out)
        b.record(stream)
        b.synchronize()
        assert r, r.to_string()
        e2e_ms.append(a.elapsed_time(b))
        e2e_admm.append(w.step_stats().admm_iterations)
    e2e_prof = w.profile(reset=True)
    e2e_val = weak_value(1, world_size, args.steps, max_over_ranks(sum(e2e_ms), "cuda"))

    # Single-GPU diagnostics: not repeated on every replica.
    variants, ref_scenes, c1 = {}, None, None
    if args.variants and world_size == 1:
        variants = variants_ab(N, torch, stream, flush, args)
        ref_scenes = reference_scenes(N, args.scene_steps)
        c1 = config1(N, torch, stream, args.cg_rel_tol, 100,
                     None if args.no_cpu_baseline else args.cpu_budget)

    if rank != 0:
        if world_size > 1:
            torch.distributed.destroy_process_group()
        return
    pk = peaks()
    cg_launch_ms = prof["cg_time_ms"] / max(prof["cg_launches"], 1)
    bytes_per_launch = prof["cg_algorithmic_bytes"] / max(prof["cg_launches"], 1)
    achieved = bytes_per_launch / (cg_launch_ms / 1e3) / 1e9 if cg_launch_ms > 0 else 0.0
    tr = traffic_per_launch()
    kernel = ("cg_dsm_cluster_kernel (persistent MAS-PCG, cluster form)"
              if cluster_solves == solves else "cg_resident / cg_kernel (persistent MAS-PCG)")
    roofline = {"bound": "hbm", "kernel": kernel,
                "achieved": round(achieved, 2), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / pk["hbm_gbs"], 5), "peak_source": pk["source"],
                "traffic": tr["bytes"] if tr else None,
                "traffic_source": (f"{tr['source']}: {tr['captured']}" if tr else None),
                "algorithmic_bytes_per_launch": round(bytes_per_launch),
                "avg_launch_ms": round(cg_launch_ms, 5),
                "cg_iterations_per_launch": round(prof["cg_iterations"] /
                                                  max(prof["cg_launches"], 1), 2),
                "cg_share_of_step": round(prof["cg_time_ms"] / total_ms, 4) if total_ms else None}
    cpu = None
    if world_size == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times, cadmm = oracle_steps(x0, v0, perm_s, offs_s, V, F, SV, SF, args.cg_rel_tol,
                                    args.steps, args.cpu_budget)
        cpu = {"value": round(len(times) / sum(times), 6), "unit": "steps/s", "cores": threads,
               "kind": "port",
               "sample": f"the first {len(times)} of the same timed steps from the same stored "
                         f"state ({sum(times):.1f} s wall, {cadmm} ADMM iterations; the GPU "
                         f"ran {sum(per_step_admm[:len(times)])} on them), OpenMP on all host "
                         f"threads"}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grid sheet + icosphere)",
        "config": bench_config(args, V, F, SV, world_size),
        "stats": {"admm_iterations_per_step": admm / args.steps,
                  "admm_iterations_per_timed_step": per_step_admm,
                  "cg_iterations_per_solve": round(cg / max(solves, 1), 2),
                  "contacts_last_step": contacts},
        "roofline": roofline, "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_val, 4), "unit": "steps/s",
                "h2d_bytes_per_step": int(SV.nbytes), "d2h_bytes_per_step": int(V.nbytes),
                "steps": args.steps, "admm_iterations_per_step": e2e_admm,
                "ms_per_step": [round(t, 1) for t in e2e_ms],
                "device_ms_per_step": [round(t, 1) for t in step_ms],
                "phases_ms_per_step": {
                    "cg_kernel_events": round(e2e_prof["cg_time_ms"] / args.steps, 2),
                    "other_admm_kernels_events": round(e2e_prof["admm_other_ms"] / args.steps, 2),
                    "admm_host_wall": round(e2e_prof["admm_host_ms"] / args.steps, 2),
                    "ccd_host_wall": round(e2e_prof["ccd_host_ms"] / args.steps, 2),
                    "dcd_host_wall": round(e2e_prof["dcd_host_ms"] / args.steps, 2),
                    "step_host_wall": round(e2e_prof["step_host_ms"] / args.steps, 2)}},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "phases_ms_per_step": {
            "cg_kernel_events": round(prof["cg_time_ms"] / args.steps, 2),
            "other_admm_kernels_events": round(prof["admm_other_ms"] / args.steps, 2),
            "contact_gs_events": round(prof["contact_gs_ms"] / args.steps, 2),
            "admm_host_wall": round(prof["admm_host_ms"] / args.steps, 2),
            "ccd_host_wall": round(prof["ccd_host_ms"] / args.steps, 2),
            "dcd_host_wall": round(prof["dcd_host_ms"] / args.steps, 2),
            "dcd_parts_host_wall": {
                k: round(prof[f"dcd_{k}_host_ms"] / args.steps, 2)
                for k in ("refit", "candidates", "build", "coloring", "layout")},
            "dcd_calls": round(prof["dcd_calls"] / args.steps, 1),
            "ccd_parts": {
                "refit_host_wall": round(prof["ccd_refit_host_ms"] / args.steps, 2),
                "candidates_host_wall": round(prof["ccd_candidates_host_ms"] / args.steps, 2),
                "first_pass_events": round(prof["ccd_first_pass_ms"] / args.steps, 2),
                "second_pass_events": round(prof["ccd_second_pass_ms"] / args.steps, 2)},
            "step_host_wall": round(prof["step_host_ms"] / args.steps, 2)},
        "variants": variants,
        "reference_scenes": ref_scenes,
        "config1": c1,
    }
    print(json.dumps(line), flush=True)
    if world_size > 1:
        torch.distributed.destroy_process_group()


RESIDENT_PHASES = ["A: p update", "barrier 1", "B: SpMV rows", "B: p.Ap block sum",
                   "barrier 2", "C: pAp total", "C: fine MAS + restriction",
                   "C: first coarse level", "C: r.z/r.r block sum + two-level z", "barrier 3",
                   "A: partial + coarse loads", "A: upper restriction chain",
                   "A: upper bank solves", "A: rz sum"]
STREAMING_PHASES = ["prolongation", "barrier 1", "SpMV", "barrier 2", "fine MAS", "barrier 3",
                    "coarse levels", "barrier 4"]
CLUSTER_PHASES = ["A: p update (own and halo)", "CTA barrier", "B: SpMV rows",
                  "B: p.Ap block sum + push", "cluster barrier 1", "C: pAp total",
                  "C: x/r update + fine MAS", "C: first-level push + r.z/r.r sum + push",
                  "cluster barrier 2", "A: halo z + totals", "A: restriction chain",
                  "A: coarse bank solves", "A: coarse r.z sum", "A: stopping test"]
FORM_NAMES = {0: "streaming", 1: "resident", 2: "cluster (redundant coarse levels)"}


def run_trace(args) -> None:
    """Median per-phase time of one CG iteration (block 0, clock64 stamps),
    over the last CG solve of one contact step from the stored state (C2) or
    of the drape's first contact step (C3)."""
    import torch

    from silk_physics_b200 import native as N

    c3 = args.trace_workload == "c3"
    V, F, SV, SF = scene_c3() if c3 else scene()
    x0, v0 = c3_start(V) if c3 else stored_state()[:2]
    stream = torch.cuda.Stream()
    opts = N.SolverOptions(fixed_linear_rel_tol=args.cg_rel_tol, profile=1, mas_bf16=args.bf16)
    w, h, _ = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    assert w.set_cloth_state(h, x0, v0)
    for _ in range(args.warmup):
        assert w.solver_step()
    assert w.set_cloth_state(h, x0, v0)
    opts.profile = 2
    assert w.set_solver_options(opts)
    assert w.solver_step()
    t = w.debug_cg_trace(h)
    ghz = t["cycles"] / max(t["ns"], 1)
    names = {0: STREAMING_PHASES, 1: RESIDENT_PHASES, 2: CLUSTER_PHASES}[t["form"]]
    med = np.median(t["phase_cycles"], axis=0)[:len(names)] / ghz / 1e3
    print(json.dumps({"cg_trace": {
        "workload": C3_WORKLOAD if c3 else WORKLOAD,
        "form": FORM_NAMES[t["form"]],
        "mas": "bf16" if args.bf16 else "fp32", "traced_iterations": t["iters"],
        "sm_ghz": round(ghz, 3), "phase_us": {n: round(float(m), 2) for n, m in zip(names, med)},
        "iteration_us": round(float(med.sum()), 2)}}), flush=True)





C5_WORKLOAD = "c5_batched_sheets_on_spheres"


def scenes_c5(count, seed=2024):
    """Independent scenes: sheet side counts log-uniform in [32, 200] (1 m
    sheets), each just above an icosphere of radius U(0.2, 0.6) m at an
    offset U([-0.3, 0.3]^2) m."""
    from silk_physics_b200 import scenes as S

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        side = int(round(math.exp(rng.uniform(math.log(32), math.log(200)))))
        r = float(rng.uniform(0.2, 0.6))
        off = rng.uniform(-0.3, 0.3, 2)
        V, F = S.grid_sheet(side, side=1.0, z=r + 0.05, jitter=1e-4,
                            seed=int(rng.integers(1 << 30)), center=(0.0, 0.0))
        SV, SF = S.icosphere(3, radius=r, center=(float(off[0]), float(off[1]), 0.0))
        out.append((V, F, SV, SF))
    return out


def run_batched(args) -> None:
    """Independent scenes stepped concurrently by silk_step_many (one CUDA
    stream per world); the batch time of a step is the latest world end event
    minus the first start event (CUDA events)."""
    import torch

    rank, local_rank, world_size = dist_env()
    torch.cuda.set_device(local_rank)
    dist_init("nccl")
    from silk_physics_b200 import native as N

    # Scenes are independent: each rank steps its share, no collective.
    scenes = shard(scenes_c5(args.c5_scenes), rank, world_size)
    opts = N.SolverOptions(fixed_linear_rel_tol=args.cg_rel_tol, mas_bf16=args.bf16)

    def build():
        ws, sts = [], []
        for V, F, SV, SF in scenes:
            st = torch.cuda.Stream()
            w, _, _ = make_world(st.cuda_stream, opts, V, F, SV, SF)
            ws.append(w)
            sts.append(st)
        for _ in range(args.c5_prelude):
            res = N.step_many(ws, 0)
            assert all(res), [r.to_string() for r in res if not r]
        return ws, sts

    nverts = sum(len(V) for V, _, _, _ in scenes)

    def timed(worlds, streams, steps, threads):
        total = 0.0
        for _ in range(steps):
            torch.cuda.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in worlds]
            for (a, _), st in zip(ev, streams):
                a.record(st)
            res = N.step_many(worlds, threads)
            for (_, b), st in zip(ev, streams):
                b.record(st)
            torch.cuda.synchronize()
            assert all(res), [r.to_string() for r in res if not r]
            total += max(ev[0][0].elapsed_time(b) for _, b in ev)
        return total

    # The same steps from the same state, concurrently and (on a second copy
    # of the worlds) one world after another.
    worlds, streams = build()
    ms = max_over_ranks(timed(worlds, streams, args.c5_steps, 0), "cuda")
    contacts = int(sum(w.step_stats().contacts for w in worlds))
    seq_ms = None
    if args.c5_sequential:
        del worlds
        worlds, streams = build()
        seq_ms = max_over_ranks(timed(worlds, streams, args.c5_steps, 1), "cuda")
    if world_size > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "scene-steps/s (independent scenes stepped concurrently)",
        "value": round(args.c5_scenes * args.c5_steps / (ms / 1e3), 4), "unit": "scene-steps/s",
        "n_gpus": world_size, "steps": args.c5_steps, "warmup": args.c5_prelude,
        "scaling": "strong", "contacts_last_step_rank0": contacts,
        "ms_per_step": round(ms / args.c5_steps, 3), "higher_is_better": True,
        "dtype": "f32", "data": "synthetic (seeded sheets + icospheres)",
        "config": {"workload": C5_WORKLOAD, "scenes": args.c5_scenes,
                   "scenes_rank0": len(worlds), "vertices_rank0": nverts,
                   "cg_rel_tol": args.cg_rel_tol, "mas": "bf16" if args.bf16 else "fp32",
                   "host_threads": "one per hardware thread"},
    }
    if seq_ms is not None:
        line["sequential_one_thread_ms_per_step"] = round(seq_ms / args.c5_steps, 3)
    print(json.dumps(line), flush=True)


def run_reference(args) -> None:
    rank, _, world_size = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    V, F, SV, SF = scene()
    x0, v0, s0, perm, offs = stored_state()
    times, admm = oracle_steps(x0, v0, perm, offs, V, F, SV, SF, args.cg_rel_tol, args.steps,
                               args.cpu_budget)
    value = len(times) / sum(times)
    sample = (f"steps {s0 + 1}-{s0 + len(times)} (the first {len(times)} of the {args.steps} "
              f"timed steps of the GPU arm) from the same stored oracle state, "
              f"{admm} ADMM iterations, OpenMP on {threads} threads; more steps than fit "
              f"{args.cpu_budget:.0f} s of CPU time are not run")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "steps/s",
        "n_gpus": world_size, "steps": len(times), "warmup": 0,
        "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grid sheet + icosphere)",
        "config": bench_config(args, V, F, SV, world_size),
        "implementation": "CPU restatement of the reference algorithm (oracle/); the reference "
                          "cannot be built offline",
        "ms_per_timed_step": [round(1e3 * t, 1) for t in times],
        "cpu_baseline": {"value": round(value, 6), "unit": "steps/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cg-rel-tol", type=float, default=1e-5,
                    help="fixed CG relative tolerance (0 = the reference's adaptive rule)")
    ap.add_argument("--bf16", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", type=int, default=1,
                    help="also the controlled A/B of the solver forms at 6.4K and 100K "
                         "vertices and the reference's example scenes")
    ap.add_argument("--variant-reps", type=int, default=5)
    ap.add_argument("--scene-steps", type=int, default=60,
                    help="steps of the cloth_ball reference scene")
    ap.add_argument("--trace-workload", choices=["c2", "c3"], default="c2")
    ap.add_argument("--batched", action="store_true",
                    help="time independent scenes stepped concurrently instead of the bench line")
    ap.add_argument("--c5-scenes", type=int, default=64)
    ap.add_argument("--c5-prelude", type=int, default=6)
    ap.add_argument("--c5-steps", type=int, default=2)
    ap.add_argument("--c5-sequential", type=int, default=1)
    ap.add_argument("--cg-trace", action="store_true",
                    help="print the CG phase breakdown of one contact step instead of the "
                         "bench line")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.cg_trace:
        run_trace(args)
    elif args.batched:
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
