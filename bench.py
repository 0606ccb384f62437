#!/usr/bin/env python
"""Benchmark: PD frames/s of the 103,680-tet beam with a moving capsule tool.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload beam|beam_mixed|batch|small]

One "step" = one PD frame (10 local/global iterations, one V-cycle each) of
the workload on one GPU.  Multi-GPU runs are independent replicas (the single
body does not shard); value = frames of all ranks / max-over-ranks time.
L2 is flushed (256 MB write) before every timed frame, outside the timed span.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PD frames/s @103,680 tets: learned+mixed vs plain FP32 MG, 1 B200, ≤1e-5·diag err"


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------
def capsule_path(frames, start=(0.0, 0.0, 3.0), dz=-0.02, sigma=0.005, half_length=4.0, seed=1):
    rng = np.random.default_rng(seed)
    c = np.array(start, np.float64)
    out = []
    for _ in range(frames):
        c = c + np.array([0.0, 0.0, dz]) + rng.normal(0.0, sigma, 3)
        out.append(((c - [half_length, 0, 0]).astype(np.float32), (c + [half_length, 0, 0]).astype(np.float32)))
    return out


def make_workload(name, mg):
    """Returns (meshes, params list, fixed masks, per-frame tool callback, description)."""
    if name in ("beam", "beam_mixed", "small"):
        dims = (4, 40, 4) if name == "small" else (12, 120, 12)
        levels = 3 if name == "small" else 4
        m = mg.box_mesh(*dims)
        fixed = (np.abs(m.positions[:, 1] - 10.0) < 1e-5).astype(np.uint8)
        p = mg.default_params(mg.SOLVER_MULTIGRID, levels=levels, iterations=10, gravity=(0.0, 0.0, 0.0))
        # Start the tool 0.3 above the top face so every timed frame has contacts.
        path = capsule_path(4096, start=(0.0, 0.0, 1.5))

        def tool(solver, f):
            a, b = path[f % len(path)]
            solver.set_capsule(a, b, 0.3)

        desc = (f"beam {dims[0]}x{dims[1]}x{dims[2]} hexes ({m.num_verts} verts, {m.num_tets} tets), "
                f"{levels} MG levels, 2+2 Jacobi sweeps, 10 PD iterations/frame, capsule r=0.3 len 8 "
                f"moving -z 0.02/frame + N(0,0.005^2) jitter (seed 1), in contact")
        return [m], [p], [fixed], tool, desc
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, nm in enumerate(names):
            if any(len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k] for r in rows):
                reasons.append(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# Algorithmic bytes per launch of the main kernels (FP32, each array once)
# ---------------------------------------------------------------------------
def coarse_vcycle_bytes(solver, params):
    """Algorithmic bytes of one k_coarse_vcycle launch (every array of every
    phase counted once; FP32 values, int32 indices, float4 vectors)."""
    L, pre, post = params.levels, params.pre_sweeps, params.post_sweeps
    lv = [solver.level_info(l) for l in range(L)]
    n = [x["n"] for x in lv]
    nnz = [x["nnz"] for x in lv]
    nch = [x["nchild"] for x in lv]
    fuse = lv[0]["fuse_l0"]
    sweep = lambda l: 8 * nnz[l] + n[l] * (16 + 16 + 8 + 16)        # ELL + e_in, r, dfull/dinv, e_out
    resid = lambda l: 8 * nnz[l] + n[l] * (16 + 16 + 4 + 16)
    restrict = lambda l: 8 * nch[l] + 16 * n[l - 1] + n[l] * (4 + 16 + 4 + 16)
    prolong = lambda l: n[l] * (16 + 16 + 16 + 16) + 16 * n[l + 1]
    b = 0
    if fuse:
        b += 8 * nnz[0] + n[0] * (16 + 16 + 4 + 16)                     # level-0 residual
        b += n[0] * (16 + 16 + 16 + 16) + 16 * n[1]                     # d += P e1
    for l in range(1, L - 1):
        b += restrict(l) + max(pre - 1, 0) * sweep(l) + resid(l) + prolong(l) + post * sweep(l)
    c = L - 1
    b += 8 * nch[c] + 16 * n[c - 1] + n[c] * 20                         # coarsest restriction
    b += 4 * n[c] * n[c] + 32 * n[c]                                     # dense inverse x r
    return float(b)


def algorithmic_bytes(kernel, solver, meshes, params):
    V = sum(m.num_verts for m in meshes)
    T = sum(m.num_tets for m in meshes)
    n0, nnz0 = solver.level_size(0)
    if kernel == "k_mg_local":
        # tet ids 16 + g vectors 40 + slot ids 16 + 4 slot writes 64; s and d 16 each per vertex
        return 136 * T + 32 * V
    if kernel == "k_l0_sweep_rg":
        # average over one V-cycle's level-0 sweeps (the first also assembles the RHS)
        plain = 56 * n0 + 8 * nnz0
        gather = plain + 16 * n0 + 4 * n0 + 16 * 4 * T   # b0, slot_ptr, slots
        k = params.pre_sweeps + params.post_sweeps
        return (gather + (k - 1) * plain) / k
    if kernel == "k_coarse_vcycle":
        return coarse_vcycle_bytes(solver, params)
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get(kernel)
    return None


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the FP64 oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_frames_per_s(meshes, params, fixeds, tool, frames, warm=1):
    from oracle.binding import Oracle
    o = Oracle(meshes[0], params[0])
    o.set_fixed(fixeds[0])
    for f in range(warm):
        tool(o, f)
        o.step()
    t0 = time.perf_counter()
    for f in range(frames):
        tool(o, warm + f)
        o.step()
    dt = time.perf_counter() - t0
    return frames / dt, dt


def run_reference(args):
    import multigridsoftbody_b200 as mg
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    meshes, params, fixeds, tool, desc = make_workload(args.workload, mg)
    cores = os.cpu_count()
    from oracle.binding import Oracle
    o = Oracle(meshes[0], params[0])
    o.set_fixed(fixeds[0])
    for f in range(args.warmup):
        tool(o, f)
        o.step()
    t0 = time.perf_counter()
    for f in range(args.steps):
        tool(o, args.warmup + f)
        o.step()
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "impl": "FP64 oracle restating the configured PD multigrid frame"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} frames of the workload after {args.warmup} warm-up frames"},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import multigridsoftbody_b200 as mg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream(device=local)
    meshes, params, fixeds, tool, desc = make_workload(args.workload, mg)
    for p in params:
        p.device = local
        p.stream = stream.cuda_stream
    solver = mg.Solver(meshes, params)
    for b, fx in enumerate(fixeds):
        solver.set_fixed(fx, body=b)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")   # 256 MB > L2

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    frame = 0
    tuned = solver.autotune(frames=5) if not args.no_tune else None
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            tool(solver, frame)
            solver.step()
            frame += 1
        solver.synchronize()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                evs[k][0].record(stream)
                tool(solver, frame)
                solver.step()
                evs[k][1].record(stream)
                frame += 1
            solver.synchronize()
        barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        # e2e: the public API with host buffers (tool pose in, positions + contacts out)
        e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
        nverts = sum(m.num_verts for m in meshes)
        for k in range(args.steps):
            flush.zero_()
            e2e_evs[k][0].record(stream)
            tool(solver, frame)
            solver.step()
            for b in range(len(meshes)):
                solver.positions(b)
                solver.contacts(b)
            e2e_evs[k][1].record(stream)
            frame += 1
        torch.cuda.synchronize()
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_evs)
        # live per-kernel profile of one frame (eager, events around every launch), cold L2
        flush.zero_()
        torch.cuda.synchronize()
        tool(solver, frame)
        prof = solver.profile_frame()
    from multigridsoftbody_b200.replicas import job_throughput, max_over_ranks
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], dist)
    value = job_throughput(args.steps, world, ms)
    e2e_value = job_throughput(args.steps, world, e2e_ms)
    if rank == 0:
        launches = solver.launches_per_frame()
        dom = max(prof.items(), key=lambda kv: kv[1][0])
        kname, (ktot, kcnt) = dom
        kavg_ms = ktot / max(kcnt, 1)
        alg = algorithmic_bytes(kname, solver, meshes, params[0])
        peak, peak_kind = measured_peaks()
        roof = None
        if alg is not None:
            ach = alg / (kavg_ms / 1e3) / 1e9
            roof = {"bound": "hbm", "kernel": kname, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "traffic": ncu_traffic(kname), "peak_kind": peak_kind,
                    "algorithmic_bytes_per_launch": alg, "avg_launch_ms": kavg_ms,
                    "share_of_frame": ktot / sum(v[0] for v in prof.values())}
        cpu = None
        if world == 1 and not args.no_cpu:
            fps, dt = cpu_frames_per_s(meshes, params, fixeds, tool, frames=args.cpu_frames)
            cpu = {"value": fps, "unit": "frames/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{args.cpu_frames} frames of the same workload, FP64 oracle ({dt:.1f} s)"}
        h2d = len(meshes) * 64 + 164          # body table + sphere set per frame
        d2h = nverts * 16 + nverts * 4        # float4 positions + contact flags
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": desc, "variant": "plain FP32 multigrid", "parallelism": f"replicas x{world}",
                           "l2": "flushed (256 MB write) before every timed frame, outside the timed span",
                           "autotuned_coarse_kernel": tuned},
                "clocks": clk.summary(),
                "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches * args.steps,
                "roofline": roof,
                "cpu_baseline": cpu,
                "kernels": {k: {"ms_per_frame": v[0], "launches": v[1]} for k, v in
                            sorted(prof.items(), key=lambda kv: -kv[1][0])}}
        print(json.dumps(line))
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="beam")
    ap.add_argument("--cpu-frames", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
