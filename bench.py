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
    """Returns (meshes, params list, fixed masks, per-frame tool callback, description,
    per-body materials or None)."""
    if name in ("beam", "beam_mixed", "small", "large_mixed"):
        dims = {"small": (4, 40, 4), "large_mixed": (24, 240, 24)}.get(name, (12, 120, 12))
        levels = {"small": 3, "large_mixed": 5}.get(name, 4)
        mixed = name in ("beam_mixed", "large_mixed")
        m = mg.box_mesh(*dims)
        fixed = (np.abs(m.positions[:, 1] - 10.0) < 1e-5).astype(np.uint8)
        p = mg.default_params(mg.SOLVER_MULTIGRID, levels=levels, iterations=10, gravity=(0.0, 0.0, 0.0),
                              precision=mg.PRECISION_MIXED if mixed else mg.PRECISION_FP32,
                              refinement_passes=2 if mixed else 1)
        # Start the tool 0.3 above the top face so every timed frame has contacts.
        path = capsule_path(4096, start=(0.0, 0.0, 1.5))

        def tool(f):
            a, b = path[f % len(path)]
            return a[None], b[None], np.array([0.3], np.float32)

        mats = None
        if name == "large_mixed":
            rng = np.random.default_rng(7)
            mats = [(np.exp(rng.uniform(np.log(5e4), np.log(2e5), m.num_tets)).astype(np.float32), 0.3)]
        desc = (f"beam {dims[0]}x{dims[1]}x{dims[2]} hexes ({m.num_verts} verts, {m.num_tets} tets), "
                f"{levels} MG levels, 2+2 Jacobi sweeps, 10 PD iterations/frame, capsule r=0.3 len 8 "
                f"moving -z 0.02/frame + N(0,0.005^2) jitter (seed 1), in contact"
                + (", mixed precision (FP64 residual, 2 refinement passes)" if mixed else "")
                + (", E log-uniform [5e4,2e5] per tet (seed 7)" if name == "large_mixed" else ""))
        return [m], [p], [fixed], tool, desc, mats
    if name == "batch":
        rng = np.random.default_rng(11)
        ns = rng.integers(2, 9, size=256)
        meshes, params, fixeds, mats = [], [], [], []
        for n in ns:
            L = 2.5 * n
            m = mg.box_mesh(int(n), int(10 * n), int(n), (-1.0, -L, -1.0), (1.0, L, 1.0))
            meshes.append(m)
            fixeds.append((np.abs(m.positions[:, 1] - L) < 1e-5).astype(np.uint8))
            params.append(mg.default_params(mg.SOLVER_MULTIGRID, levels=3, iterations=10, gravity=(0.0, 0.0, 0.0)))
            E = float(np.exp(rng.uniform(np.log(5e4), np.log(2e5))))
            nu = float(rng.uniform(0.25, 0.45))
            mats.append((np.full(m.num_tets, E, np.float32), nu))
        start = np.array([0.0, 0.0, 1.15]) + rng.uniform(-0.5, 0.5, (256, 3))
        vel = np.random.default_rng(12)

        traj = [start]
        for _ in range(4096):
            traj.append(traj[-1] + vel.normal(0.0, 0.01, (256, 3)))

        def tool(f):
            c = traj[f % len(traj)]
            return ((c - [2.0, 0, 0]).astype(np.float32), (c + [2.0, 0, 0]).astype(np.float32),
                    np.full(256, 0.2, np.float32))

        V = sum(m.num_verts for m in meshes)
        T = sum(m.num_tets for m in meshes)
        desc = (f"batch of 256 beams n x 10n x n hexes, n~U{{2..8}} (seed 11): {V} verts, {T} tets in total; "
                f"E log-uniform [5e4,2e5], nu U[0.25,0.45] per body; capsule r=0.2 len 4 per body, start "
                f"(0,0,1.15)+U(-0.5,0.5)^3, velocity N(0,0.01^2)/axis/frame; 3 levels, 10 PD iterations; one launch per phase")
        return meshes, params, fixeds, tool, desc, mats
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
def apply_tool(solver, poses):
    a, b, r = poses
    if len(r) == 1:
        solver.set_capsule(a[0], b[0], float(r[0]))
    else:
        solver.set_capsules(a, b, r)


def make_oracles(meshes, params, fixeds, mats):
    from oracle.binding import Oracle
    out = []
    for i, m in enumerate(meshes):
        o = Oracle(m, params[i])
        o.set_fixed(fixeds[i])
        if mats is not None:
            o.set_material(*mats[i])
        out.append(o)
    return out


def oracle_frames(oracles, tool, f0, frames):
    for f in range(f0, f0 + frames):
        a, b, r = tool(f)
        for i, o in enumerate(oracles):
            o.set_capsule(a[i], b[i], float(r[i]))
            o.step()


def cpu_frames_per_s(meshes, params, fixeds, tool, mats, frames, warm=1):
    os_ = make_oracles(meshes, params, fixeds, mats)
    oracle_frames(os_, tool, 0, warm)
    t0 = time.perf_counter()
    oracle_frames(os_, tool, warm, frames)
    dt = time.perf_counter() - t0
    return frames / dt, dt


def run_reference(args):
    import multigridsoftbody_b200 as mg
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    meshes, params, fixeds, tool, desc, mats = make_workload(args.workload, mg)
    cores = os.cpu_count()
    os_ = make_oracles(meshes, params, fixeds, mats)
    oracle_frames(os_, tool, 0, args.warmup)
    t0 = time.perf_counter()
    oracle_frames(os_, tool, args.warmup, args.steps)
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
    meshes, params, fixeds, tool, desc, mats = make_workload(args.workload, mg)
    for p in params:
        p.device = local
        p.stream = stream.cuda_stream
    solver = mg.Solver(meshes, params)
    for b, fx in enumerate(fixeds):
        solver.set_fixed(fx, body=b)
        if mats is not None:
            solver.set_material(*mats[b], body=b)
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
            apply_tool(solver, tool(frame))
            solver.step()
            frame += 1
        solver.synchronize()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                evs[k][0].record(stream)
                apply_tool(solver, tool(frame))
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
            apply_tool(solver, tool(frame))
            solver.step()
            solver.all_positions()
            solver.all_contact_flags()
            e2e_evs[k][1].record(stream)
            frame += 1
        torch.cuda.synchronize()
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_evs)
        # live per-kernel profile of one frame (eager, events around every launch), cold L2
        flush.zero_()
        torch.cuda.synchronize()
        apply_tool(solver, tool(frame))
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
            fps, dt = cpu_frames_per_s(meshes, params, fixeds, tool, mats, frames=args.cpu_frames)
            cpu = {"value": fps, "unit": "frames/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{args.cpu_frames} frames of the same workload, FP64 oracle ({dt:.1f} s)"}
        h2d = len(meshes) * 88 + 164          # body table (88 B per body) + sphere set per frame
        d2h = nverts * 16 + nverts * 4        # float4 positions + contact flags
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": desc, "variant": "mixed precision multigrid" if params[0].precision == 1 else "plain FP32 multigrid", "parallelism": f"replicas x{world}",
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
