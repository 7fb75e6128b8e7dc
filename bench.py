#!/usr/bin/env python
"""Benchmark of the per-step cloth pipeline (silk::World::solver_step).

Workload (N = 1): the 6.4K-vertex sheet of the benchmark's second
configuration -- an 80 x 80 grid (12,482 triangles, side 1 m, jitter
N(0, 1e-4) m from a fixed seed) dropped from z = 1 onto a static icosphere
(subdivision 4, radius 0.3 m), self-collision and obstacle CCD on, float32,
dt = 1/60, gravity -9.81.  A step is one solver_step.  The sheet first falls
freely for `--prelude` untimed steps so that the timed steps run with active
contacts (the regime the reference's "6K cloth with active collision" claim
describes); then `--warmup` untimed and `--steps` timed steps follow.

Metric: steps/s (higher is better).  `value` is device time (CUDA events on
the world's stream) with inputs resident; `e2e` drives the public API with
host buffers each step (obstacle position upload + solver_step + position
readback).  Between timed steps a 256 MiB buffer is written to flush L2.

Multi-GPU: scenes are independent, so --gpus N runs N replicas (one process
per GPU, no collective on the data path; barrier + max over ranks only).

`--impl reference` times the CPU restatement of the reference algorithm
(oracle/, the reference itself cannot be built here) on all host cores on the
same scene and steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOAD = "c2_sheet80_on_icosphere_r0.3"
METRIC = "steps/s (6.4K-vertex sheet on sphere, active contact)"


def scene(seed=1236):
    from silk_physics_b200 import scenes as S

    V, F = S.grid_sheet(80, side=1.0, z=1.0, jitter=1e-4, seed=seed)
    SV, SF = S.icosphere(4, radius=0.3)
    return V, F, SV, SF


C3_WORKLOAD = "c3_sheet316_on_icosphere_r0.6"
MODEL = ROOT / "silk_physics_b200" / "models" / "warm_start.npy"


def scene_c3(seed=1237):
    from silk_physics_b200 import scenes as S

    V, F = S.grid_sheet(316, side=2.0, z=0.7, jitter=1e-4, seed=seed)
    SV, SF = S.icosphere(4, radius=0.6)
    return V, F, SV, SF


def timed_variant(N, torch, stream, flush, V, F, SV, SF, cg_rel_tol, bf16, learned,
                  prelude, steps, extrap=False):
    """Steps/s and CG statistics of one solver variant on one scene: `prelude`
    untimed steps, then `steps` steps timed with CUDA events (L2 flushed
    between steps)."""
    opts = N.SolverOptions(fixed_linear_rel_tol=cg_rel_tol, profile=True, mas_bf16=bf16,
                           learned_warm_start=learned, admm_extrapolated_start=extrap)
    w, h, _ = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    if learned:
        from silk_physics_b200 import learned as L

        r = w.set_warm_start_model(L.load(str(MODEL)))
        assert r, r.to_string()
    for _ in range(prelude):
        r = w.solver_step()
        assert r, r.to_string()
    w.profile(reset=True)
    ms, admm, cg, solves, first, taken, outer, ext = 0.0, 0, 0, 0, 0, 0, 0, 0
    for k in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xff)
            a.record(stream)
        r = w.solver_step()
        b.record(stream)
        b.synchronize()
        assert r, r.to_string()
        ms += a.elapsed_time(b)
        st = w.step_stats()
        admm += st.admm_iterations
        cg += st.cg_iterations
        solves += st.cg_solves
        first += st.cg_first_solve_iterations
        taken += st.learned_starts
        ext += st.extrapolated_starts
        outer += st.outer_iterations
    prof = w.profile(reset=True)
    return {"value": round(steps / (ms / 1e3), 4), "ms_per_step": round(ms / steps, 3),
            "cg_kernel_ms_per_step": round(prof["cg_time_ms"] / steps, 2),
            "other_admm_kernels_ms_per_step": round(prof["admm_other_ms"] / steps, 2),
            "contact_gs_ms_per_step": round(prof["contact_gs_ms"] / steps, 2),
            "ccd_host_ms_per_step": round(prof["ccd_host_ms"] / steps, 2),
            "dcd_host_ms_per_step": round(prof["dcd_host_ms"] / steps, 2),
            "admm_iterations_per_step": admm / steps,
            "cg_iterations_per_solve": round(cg / max(solves, 1), 2),
            "first_solve_cg_iterations_per_outer": round(first / max(outer, 1), 2),
            "learned_starts_taken": taken, "extrapolated_starts_taken": ext,
            "outer_iterations": outer}


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
    """DRAM bytes per CG launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "cg_resident_c2.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def make_world(stream_handle, opts, V, F, SV, SF):
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
    return w, h, hs


def cpu_oracle_sample(x0, v0, V, F, SV, SF, cg_rel_tol, budget_s=20.0):
    """Time the CPU restatement from the same state on all host cores.

    Contact steps of this algorithm take minutes on a CPU, so the sample is
    the steps that fit in ~budget_s (at least one); the result is steps/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    ow = pyoracle.OracleWorld(config=dict(acceleration=(0.0, 0.0, -9.81),
                                          fixed_linear_rel_tol=cg_rel_tol))
    nv = len(V)
    perm = np.arange(nv, dtype=np.int32)
    offs = np.unique(np.append(np.arange(0, nv, 32), nv)).astype(np.int32)
    h = ow.add_cloth(V, F, [], perm, offs)
    ow.add_obstacle(SV, SF)
    ow.set_state(h, x0, v0)
    t0 = time.perf_counter()
    steps = 0
    admm = 0
    while True:
        ow.step()
        steps += 1
        admm += ow.stats()["admm_iterations"]
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return steps / el, steps, el, admm


def run_ours(args) -> None:
    import torch

    rank, local_rank, world_size = dist_env()
    torch.cuda.set_device(local_rank)
    dist_init("nccl")
    from silk_physics_b200 import native as N

    V, F, SV, SF = scene()
    stream = torch.cuda.Stream()
    opts = N.SolverOptions(fixed_linear_rel_tol=args.cg_rel_tol, profile=True,
                           mas_bf16=args.bf16)
    w, h, hs = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    x = np.zeros(V.size, np.float32)
    for _ in range(args.prelude):
        r = w.solver_step()
        assert r, r.to_string()
    for _ in range(args.warmup):
        r = w.solver_step()
        assert r, r.to_string()
    state_x = np.zeros(V.size, np.float32)
    state_v = np.zeros(V.size, np.float32)
    w.get_cloth_position(h, state_x)
    w.get_cloth_velocity(h, state_v)
    w.profile(reset=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = admm = cg = solves = contacts = admm_first = ccd_first = 0
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
            if k < args.e2e_steps:
                admm_first += st.admm_iterations
                ccd_first += st.ccd_queries
            cg += st.cg_iterations
            solves += st.cg_solves
            contacts = st.contacts
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    prof = w.profile(reset=True)
    total_ms = max_over_ranks(total_ms, "cuda")
    value = weak_value(1, world_size, args.steps, total_ms)

    # Learned warm start + BF16 MAS on the same scene, and the 100K-vertex
    # sheet (plain FP32 vs learned + BF16), each from its own fresh world.
    variants = {}
    # Single-GPU diagnostics: not repeated on every replica.
    if args.variants and MODEL.exists() and world_size == 1:
        for name, bf16, learned, extrap in (("c2_bf16", True, False, False),
                                            ("c2_learned_bf16", True, True, False),
                                            ("c2_extrapolated", False, False, True),
                                            ("c2_learned_extrapolated_bf16", True, True, True)):
            variants[name] = timed_variant(N, torch, stream, flush, V, F, SV, SF,
                                           args.cg_rel_tol, bf16, learned,
                                           args.prelude + args.warmup, args.variant_steps,
                                           extrap)
        V3, F3, SV3, SF3 = scene_c3()
        c3 = {"workload": C3_WORKLOAD, "vertices": int(len(V3)), "faces": int(len(F3)),
              "prelude_steps": args.c3_prelude, "steps": args.c3_steps}
        for name, bf16, learned, extrap in (("plain_fp32", False, False, False),
                                            ("bf16", True, False, False),
                                            ("learned_bf16", True, True, False),
                                            ("learned_extrapolated_bf16", True, True, True)):
            c3[name] = timed_variant(N, torch, stream, flush, V3, F3, SV3, SF3, args.cg_rel_tol,
                                     bf16, learned, args.c3_prelude, args.c3_steps, extrap)
        for name in ("learned_bf16", "learned_extrapolated_bf16"):
            c3[name + "_over_plain"] = round(c3[name]["value"] / c3["plain_fp32"]["value"], 3)
        variants["c3"] = c3

    # End to end through the public API with host buffers, on the same steps:
    # a fresh world replays the prelude and warm-up (the step is
    # deterministic), then the first e2e_steps timed steps run with the
    # obstacle position uploaded from pinned host memory and the cloth
    # position read back to it inside the timed region.
    we, he, hse = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    for _ in range(args.prelude + args.warmup):
        r = we.solver_step()
        assert r, r.to_string()
    pin_obs = torch.from_numpy(SV.ravel().copy()).pin_memory().numpy()
    pin_out = torch.empty(V.size, dtype=torch.float32).pin_memory().numpy()
    e2e_ms = []
    e2e_admm = e2e_ccd = 0
    we.profile(reset=True)
    n_e2e = min(args.e2e_steps, args.steps)
    for k in range(n_e2e):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(k & 0xff)
        a.record(stream)
        we.set_obstacle_position(hse, pin_obs)
        r = we.solver_step()
        we.get_cloth_position(he, pin_out)
        b.record(stream)
        b.synchronize()
        assert r, r.to_string()
        e2e_ms.append(a.elapsed_time(b))
        e2e_admm += we.step_stats().admm_iterations
        e2e_ccd += we.step_stats().ccd_queries
    e2e_prof = we.profile(reset=True)
    # Every rank takes both reductions, in this order.
    e2e_val = weak_value(1, world_size, n_e2e, max_over_ranks(sum(e2e_ms), "cuda"))
    value_same_steps = weak_value(1, world_size, n_e2e,
                                  max_over_ranks(sum(step_ms[:n_e2e]), "cuda"))
    del we

    if rank != 0:
        if world_size > 1:
            torch.distributed.destroy_process_group()
        return
    pk = peaks()
    cg_launch_ms = prof["cg_time_ms"] / max(prof["cg_launches"], 1)
    bytes_per_launch = prof["cg_algorithmic_bytes"] / max(prof["cg_launches"], 1)
    achieved = bytes_per_launch / (cg_launch_ms / 1e3) / 1e9 if cg_launch_ms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": "cg_resident_cluster_kernel (persistent MAS-PCG)",
                "achieved": round(achieved, 2), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / pk["hbm_gbs"], 5), "peak_source": pk["source"],
                "traffic": traffic_per_launch(),
                "algorithmic_bytes_per_launch": round(bytes_per_launch),
                "avg_launch_ms": round(cg_launch_ms, 5),
                "cg_share_of_step": round(prof["cg_time_ms"] / total_ms, 4) if total_ms else None}
    cpu = None
    if world_size == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sps, n, el, cadmm = cpu_oracle_sample(state_x, state_v, V, F, SV, SF,
                                               args.cg_rel_tol, args.cpu_budget)
        cpu = {"value": round(sps, 6), "unit": "steps/s", "cores": threads, "kind": "port",
               "sample": f"{n} step(s) of the same scene from the GPU state after "
                         f"{args.prelude + args.warmup} steps, {el:.1f} s wall, "
                         f"{cadmm} ADMM iterations, OpenMP on all host threads"}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grid sheet + icosphere)",
        "config": {"workload": WORKLOAD, "vertices": int(len(V)), "faces": int(len(F)),
                   "obstacle_vertices": int(len(SV)), "prelude_steps": args.prelude,
                   "cg_rel_tol": args.cg_rel_tol if args.cg_rel_tol > 0 else "adaptive (reference)",
                   "mas": "bf16" if args.bf16 else "fp32",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "admm_iterations_per_step": admm / args.steps,
                   "cg_iterations_per_solve": round(cg / max(solves, 1), 2),
                   "contacts_last_step": contacts,
                   "parallelism": f"replicas x{world_size}"},
        "roofline": roofline, "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_val, 4), "unit": "steps/s",
                "h2d_bytes_per_step": int(SV.nbytes), "d2h_bytes_per_step": int(V.nbytes),
                "steps": n_e2e, "device_value_same_steps": round(value_same_steps, 4),
                "admm_iterations": e2e_admm, "device_admm_iterations_same_steps": admm_first,
                # set_obstacle_position marks the obstacle as moving (as the
                # reference does), so the e2e steps run the moving-obstacle
                # collision path: its CCD queries beside the device run's.
                "ccd_queries": e2e_ccd, "device_ccd_queries_same_steps": ccd_first,
                "ms_per_step": [round(t, 1) for t in e2e_ms],
                "device_ms_per_step": [round(t, 1) for t in step_ms[:n_e2e]],
                "phases_ms_per_step": {
                    "cg_kernel_events": round(e2e_prof["cg_time_ms"] / n_e2e, 2),
                    "other_admm_kernels_events": round(e2e_prof["admm_other_ms"] / n_e2e, 2),
                    "admm_host_wall": round(e2e_prof["admm_host_ms"] / n_e2e, 2),
                    "ccd_host_wall": round(e2e_prof["ccd_host_ms"] / n_e2e, 2),
                    "dcd_host_wall": round(e2e_prof["dcd_host_ms"] / n_e2e, 2),
                    "step_host_wall": round(e2e_prof["step_host_ms"] / n_e2e, 2)}},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "phases_ms_per_step": {
            "cg_kernel_events": round(prof["cg_time_ms"] / args.steps, 2),
            "other_admm_kernels_events": round(prof["admm_other_ms"] / args.steps, 2),
            "contact_gs_events": round(prof["contact_gs_ms"] / args.steps, 2),
            "admm_host_wall": round(prof["admm_host_ms"] / args.steps, 2),
            "ccd_host_wall": round(prof["ccd_host_ms"] / args.steps, 2),
            "dcd_host_wall": round(prof["dcd_host_ms"] / args.steps, 2),
            "step_host_wall": round(prof["step_host_ms"] / args.steps, 2)},
        "variants": variants,
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


def run_trace(args) -> None:
    """Median per-phase time of one CG iteration (block 0, clock64 stamps)."""
    import torch

    from silk_physics_b200 import native as N

    c3 = args.trace_workload == "c3"
    V, F, SV, SF = scene_c3() if c3 else scene()
    stream = torch.cuda.Stream()
    opts = N.SolverOptions(fixed_linear_rel_tol=args.cg_rel_tol, profile=1, mas_bf16=args.bf16)
    w, h, _ = make_world(stream.cuda_stream, opts, V, F, SV, SF)
    for _ in range(args.prelude + args.warmup):
        assert w.solver_step()
    opts.profile = 2
    assert w.set_solver_options(opts)
    assert w.solver_step()
    t = w.debug_cg_trace(h)
    ghz = t["cycles"] / max(t["ns"], 1)
    names = RESIDENT_PHASES if t["form"] == 1 else STREAMING_PHASES
    med = np.median(t["phase_cycles"], axis=0)[:len(names)] / ghz / 1e3
    print(json.dumps({"cg_trace": {
        "workload": C3_WORKLOAD if c3 else WORKLOAD,
        "steps_before": args.prelude + args.warmup,
        "form": "resident" if t["form"] == 1 else "streaming",
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
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    V, F, SV, SF = scene()
    ow = pyoracle.OracleWorld(config=dict(acceleration=(0.0, 0.0, -9.81),
                                          fixed_linear_rel_tol=args.cg_rel_tol))
    nv = len(V)
    perm = np.arange(nv, dtype=np.int32)
    offs = np.unique(np.append(np.arange(0, nv, 32), nv)).astype(np.int32)
    h = ow.add_cloth(V, F, [], perm, offs)
    ow.add_obstacle(SV, SF)
    # The oracle's own state after the default 24 prelude + 3 warm-up steps
    # (oracle/make_reference_state.py) spares replaying them on the host
    # cores; further untimed steps run from there when more are asked for.
    state = ROOT / "oracle" / "reference_state_c2_step27.npz"
    start = args.prelude + args.warmup
    done = 0
    if args.cg_rel_tol == 1e-5 and start >= 27 and state.exists():
        st = np.load(state)
        ow.set_state(h, st["x"], st["v"])
        done = int(st["steps"])
    t_pre = time.perf_counter()
    for _ in range(start - done):
        ow.step()
    pre = time.perf_counter() - t_pre
    times = []
    admm = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a = time.perf_counter()
        ow.step()
        times.append(time.perf_counter() - a)
        admm += ow.stats()["admm_iterations"]
        if time.perf_counter() - t0 > args.cpu_budget and len(times) >= 1:
            break
    value = len(times) / sum(times)
    origin = (f"from the oracle's stored state after {done} steps, "
              f"{start - done} more untimed" if done else f"after {start} untimed steps")
    sample = (f"{len(times)} timed step(s) {origin} ({pre:.1f} s), {admm} ADMM iterations, "
              f"OpenMP on {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "steps/s",
        "n_gpus": world_size, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grid sheet + icosphere)",
        "config": {"workload": WORKLOAD, "vertices": int(nv), "prelude_steps": args.prelude,
                   "implementation": "CPU restatement of the reference algorithm (oracle/); "
                                     "the reference cannot be built offline"},
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
    ap.add_argument("--prelude", type=int, default=24)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cg-rel-tol", type=float, default=1e-5,
                    help="fixed CG relative tolerance (0 = the reference's adaptive rule)")
    ap.add_argument("--bf16", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", type=int, default=1,
                    help="also time learned + BF16 MAS at 6.4K and plain vs learned + BF16 "
                         "at 100K vertices (needs the trained model file)")
    ap.add_argument("--variant-steps", type=int, default=5)
    ap.add_argument("--c3-prelude", type=int, default=8)
    ap.add_argument("--c3-steps", type=int, default=2)
    ap.add_argument("--trace-workload", choices=["c2", "c3"], default="c2")
    ap.add_argument("--batched", action="store_true",
                    help="time independent scenes stepped concurrently instead of the bench line")
    ap.add_argument("--c5-scenes", type=int, default=64)
    ap.add_argument("--c5-prelude", type=int, default=6)
    ap.add_argument("--c5-steps", type=int, default=2)
    ap.add_argument("--c5-sequential", type=int, default=1)
    ap.add_argument("--cg-trace", action="store_true",
                    help="print the CG phase breakdown of one step (after prelude and warm-up) "
                         "instead of the bench line")
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
