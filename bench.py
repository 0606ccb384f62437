#!/usr/bin/env python
"""Benchmark: PD frames/s of the 103,680-tet beam with a moving capsule tool.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload beam|beam_plain|beam_mixed|large_mixed|batch|blob|small]

One "step" = one PD frame (10 local/global iterations) of the workload on one
GPU.  The default workload is the headline: the learned-smoother mixed-precision
multigrid (1 refinement pass per PD iteration) on the 103,680-tet beam, with
the plain FP32 multigrid (1 and 2 V-cycles per PD iteration) timed the same way
in the same run and all checked for max vertex error against a converged
reference; the ratio that counts is against the plain form that meets the
1e-5 x bbox-diagonal bar.
Multi-GPU runs are independent replicas (the single body does not shard);
value = frames of all ranks / max-over-ranks time.  L2 is flushed (256 MB
write) before every timed frame, outside the timed span.
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
    if name in ("beam", "beam_plain", "beam_mixed", "small", "large_mixed"):
        dims = {"small": (4, 40, 4), "large_mixed": (24, 240, 24)}.get(name, (12, 120, 12))
        levels = {"small": 3, "large_mixed": 5}.get(name, 4)
        mixed = name in ("beam", "beam_mixed", "large_mixed")
        m = mg.box_mesh(*dims)
        fixed = (np.abs(m.positions[:, 1] - 10.0) < 1e-5).astype(np.uint8)
        p = mg.default_params(mg.SOLVER_MULTIGRID, levels=levels, iterations=10, gravity=(0.0, 0.0, 0.0),
                              precision=mg.PRECISION_MIXED if mixed else mg.PRECISION_FP32,
                              refinement_passes=(1 if name == "beam" else 2) if mixed else 1)
        # The tool starts 0.3 above the top face so every timed frame has contacts: frames 75-300 of the
        # configured 300-frame path (z from 1.5 down to -3), repeated, so the timed states stay within it.
        path = capsule_path(225, start=(0.0, 0.0, 1.5))

        def tool(f):
            a, b = path[f % len(path)]
            return a[None], b[None], np.array([0.3], np.float32)

        mats = None
        if name == "large_mixed":
            rng = np.random.default_rng(7)
            mats = [(np.exp(rng.uniform(np.log(5e4), np.log(2e5), m.num_tets)).astype(np.float32), 0.3)]
        desc = (f"beam {dims[0]}x{dims[1]}x{dims[2]} hexes ({m.num_verts} verts, {m.num_tets} tets), "
                f"{levels} MG levels, 10 PD iterations/frame, capsule r=0.3 len 8 "
                f"moving -z 0.02/frame + N(0,0.005^2) jitter (seed 1), in contact (frames 75-300 of the configured path, repeated)"
                + (", learned smoother (1 learned sweep before and after the coarse correction, residual guard "
                   "with plain fallback)" if name == "beam" else ", 2+2 Jacobi sweeps")
                + ((", mixed precision (FP64 residual, %d refinement pass%s)" % (p.refinement_passes,
                                                                                "" if p.refinement_passes == 1 else "es"))
                   if mixed else "")
                + (", E log-uniform [5e4,2e5] per tet (seed 7)" if name == "large_mixed" else ""))
        return [m], [p], [fixed], tool, desc, mats
    if name == "blob":
        from multigridsoftbody_b200.learned import blob_scene, blob_tool_path
        m, fixed, p = blob_scene(precision=mg.PRECISION_MIXED, refinement_passes=1)
        path = blob_tool_path(300, seed=1)   # 300 frames as config 1's tool path, repeated

        def tool(f):
            a, b = path[f % len(path)]
            return a[None], b[None], np.array([0.3], np.float32)

        desc = (f"organ-like blob 64x32x48 voxels at 0.25 m ({m.num_verts} verts, {m.num_tets} tets), fixed x<-5, "
                f"E 3e4, nu 0.45, gravity -z, 5 MG levels, 10 PD iterations, capsule r=0.3 len 8 from (0,0,3.3) "
                f"moving -z 0.02/frame + jitter (seed 1); learned smoother + mixed precision (1 refinement pass)")
        return [m], [p], [fixed], tool, desc, None
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

        traj = [start]   # the configured 200 frames, repeated
        for _ in range(199):
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


def shard_workload(meshes, params, fixeds, tool, mats, world, rank):
    """This rank's share of a workload: a batch of bodies is split by body (greedy by tet count, no
    collective on the data path); a single body runs as a replica on every rank.  Returns the rank's
    meshes, params, fixed masks, tool callback, materials and the BodyShard (None for replicas)."""
    from multigridsoftbody_b200.replicas import BodyShard
    if world <= 1 or len(meshes) <= 1:
        return meshes, params, fixeds, tool, mats, None
    shard = BodyShard([m.num_tets for m in meshes], world, rank)
    return (shard.take(meshes), shard.take(params), shard.take(fixeds), shard.tool(tool), shard.take(mats),
            shard)


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
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # start timing only once the sampler is running (its first line is out)
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None and os.path.getsize(self.path) == 0:
                time.sleep(0.01)
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
class LevelBytes:
    """Algorithmic bytes of one launch of each multigrid phase on level l
    (every array counted once; FP32 values, int32 indices, float4 vectors)."""

    def __init__(self, solver, params):
        self.L, self.pre, self.post = params.levels, params.pre_sweeps, params.post_sweeps
        lv = [solver.level_info(l) for l in range(self.L)]
        self.n = [x["n"] for x in lv]
        self.nnz = [x["nnz"] for x in lv]
        self.nch = [x["nchild"] for x in lv]
        self.fuse = lv[0]["fuse_l0"]
        self.split = solver.coarse_split()
        # the coarsest level is a dense inverse per body: sum of the bodies' n^2
        self.dense = sum(solver.body_level_size(b, self.L - 1) ** 2 for b in range(solver.num_bodies))

    def sweep(self, l):      # ELL + e_in, r, dfull/dinv, e_out
        return 8 * self.nnz[l] + self.n[l] * (16 + 16 + 8 + 16)

    def resid(self, l):      # ELL + e, r, dfull, res
        return 8 * self.nnz[l] + self.n[l] * (16 + 16 + 4 + 16)

    def restrict(self, l):   # children (id, weight) + finer residual; r, e, dinv written/read
        return 8 * self.nch[l] + 16 * self.n[l - 1] + self.n[l] * (4 + 16 + 4 + 16)

    def prolong(self, l):    # level l: parents ids/weights, cur, dst; coarser correction
        return self.n[l] * (16 + 16 + 16 + 16) + 16 * self.n[l + 1]

    def grid_levels(self):
        return range(1, self.split)

    def coarse_vcycle(self):
        """One launch of the cluster kernel: levels split..L-1."""
        L, pre, post = self.L, self.pre, self.post
        b = 0
        if self.fuse:
            b += self.resid(0) + self.prolong(0)
        for l in range(self.split, L - 1):
            b += self.restrict(l) + max(pre - 1, 0) * self.sweep(l) + self.resid(l) + self.prolong(l) + post * self.sweep(l)
        c = L - 1
        b += 8 * self.nch[c] + 16 * self.n[c - 1] + self.n[c] * 20       # coarsest restriction
        b += 4 * self.dense + 32 * self.n[c]                             # dense inverses x r
        return float(b)

    def mean_over_grid_levels(self, f, per_level):
        tot = sum(per_level * f(l) for l in self.grid_levels())
        cnt = per_level * len(self.grid_levels())
        return float(tot / cnt) if cnt else None


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
    lb = LevelBytes(solver, params)
    if kernel == "k_coarse_vcycle":
        return lb.coarse_vcycle()
    if kernel == "k_l0_residual_rg":
        return float(lb.resid(0))
    if kernel == "k_l0_prolong":
        return float(lb.prolong(0))
    if kernel == "k_lvl_sweep":        # (pre - 1) + post sweeps on each grid-wide level
        return lb.mean_over_grid_levels(lb.sweep, max(params.pre_sweeps - 1, 0) + params.post_sweeps)
    if kernel == "k_lvl_residual":
        return lb.mean_over_grid_levels(lb.resid, 1)
    if kernel == "k_lvl_restrict":
        return lb.mean_over_grid_levels(lb.restrict, 1)
    if kernel == "k_lvl_prolong":
        return lb.mean_over_grid_levels(lb.prolong, 1)
    if kernel.startswith("k_ls_guard_residual"):
        # residual check: e, b 32 B + D, fix 8 B per row, 8 B/nnz; mixed precision also updates the
        # FP64 displacement (read + write 64 B) and its FP32 mirror (16 B)
        mixed = params.precision == 1
        return (40 + (80 if mixed else 0)) * n0 + 8 * nnz0
    if kernel == "k_mx_residual":
        # FP64 outer residual: ELL value 8 + column 4 B per entry; per row the FP64 displacement (32), diagonal
        # (8), contact weight, Jacobi weight, fix flag (12), r32 and e out (32), the learned start residual (16)
        # and the right-hand side: read (32) or, in a PD iteration's first pass, assembled from b0 (32) and the
        # row's slots (64 B per tet over the body) and written (32)
        per_row = 32 + 8 + 12 + 32 + 16
        first = 32 + 32 + 4 + 64 * T / max(n0, 1)
        k = max(params.refinement_passes, 1)
        return 12 * nnz0 + n0 * (per_row + (first + (k - 1) * 32) / k)
    if kernel == "k_ls_sweep_tc":
        # learned sweep: level-0 row walk (8 B/nnz, r/D/L/fix 28 B per row) + d read/write 32 B per row;
        # the 12.9 KB weight image per CTA comes from L2
        return 60 * n0 + 8 * nnz0
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# the mesh each workload runs; ncu DRAM traffic is recorded per (mesh, kernel) in profiles/ncu_traffic.json
TRAFFIC_MESH = {"beam": "beam12x120x12", "beam_plain": "beam12x120x12", "beam_mixed": "beam12x120x12"}


def ncu_traffic(kernel, workload):
    """DRAM bytes (read + write) per launch of `kernel` from an ncu capture of the workload's mesh, or
    None when no capture of that mesh exists."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    mesh = TRAFFIC_MESH.get(workload)
    if mesh is None or not os.path.exists(p):
        return None
    return json.load(open(p)).get("meshes", {}).get(mesh, {}).get(kernel)


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


def cpu_frames_per_s(meshes, params, fixeds, tool, mats, frames, seconds, warm=1):
    """Oracle frames of the workload after `warm` warm-up frames, until `seconds` have passed (at least
    3 frames, at most `frames`): (frames/s, frames, seconds)."""
    os_ = make_oracles(meshes, params, fixeds, mats)
    oracle_frames(os_, tool, 0, warm)
    t0 = time.perf_counter()
    n = 0
    while n < frames and (n < 3 or time.perf_counter() - t0 < seconds):
        oracle_frames(os_, tool, warm + n, 1)
        n += 1
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def cpu_baseline(meshes, wparams, fixeds, tool, mats, args, at_bar_key=None):
    """The FP64 oracle of the workload's configured plain iteration on all host threads (`value`) and on
    one thread, plus, when the plain FP32 form that meets the error bar differs from the configured one,
    the oracle running that form on all threads (the configured 1-V-cycle iteration misses the bar on
    the headline scene)."""
    from oracle.binding import set_threads
    from multigridsoftbody_b200 import sweeps as sw
    p0 = wparams[0]
    form = f"{p0.pre_sweeps}+{p0.post_sweeps} sweeps, {p0.refinement_passes} V-cycle(s) per PD iteration"
    cores = set_threads(0)
    fps, nfr, dt = cpu_frames_per_s(meshes, wparams, fixeds, tool, mats, frames=args.cpu_frames,
                                    seconds=args.cpu_seconds)
    out = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
           "sample": f"{nfr} frames of the same workload ({dt:.1f} s), FP64 oracle of its configured plain "
                     f"iteration ({form}); on the headline scene that iteration misses the 1e-5 x diag bar"}
    set_threads(1)
    f1, n1, d1 = cpu_frames_per_s(meshes, wparams, fixeds, tool, mats, frames=args.cpu_frames,
                                  seconds=args.cpu_seconds / 2)
    out["single_thread"] = {"value": f1, "cores": 1, "sample": f"{n1} frames ({d1:.1f} s), same iteration"}
    set_threads(0)
    if at_bar_key:
        sweeps = tuple(int(v) for v in at_bar_key.rsplit("_", 1)[1].split("+"))
        passes = int(at_bar_key.split("_")[2].replace("pass", ""))
        pb = [sw.variant_params(p, sweeps, passes, False) for p in wparams]
        fb, nb, db = cpu_frames_per_s(meshes, pb, fixeds, tool, mats, frames=args.cpu_frames,
                                      seconds=args.cpu_seconds / 2)
        out["at_bar_form"] = {"value": fb, "cores": cores, "form": at_bar_key.replace("plain_fp32", "oracle_fp64"),
                              "sample": f"{nb} frames ({db:.1f} s), the FP64 oracle running the plain form that "
                                        f"meets the bar on the GPU"}
    return out


def run_reference(args):
    import multigridsoftbody_b200 as mg
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.binding import set_threads
    cores = set_threads(0)
    if args.workload == "twolevel":
        from oracle.binding import OracleTwoLevel
        coarse, fine, cf, ff, p, sphere, desc = twolevel_scene(mg)
        o = OracleTwoLevel(coarse, fine, p)
        o.set_fixed(cf, ff)
        for f in range(args.warmup):
            o.set_spheres(*sphere(f))
            o.step()
        t0 = time.perf_counter()
        for k in range(args.steps):
            o.set_spheres(*sphere(args.warmup + k))
            o.step()
        dt = time.perf_counter() - t0
        v = args.steps / dt
        print(json.dumps({"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": 0, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": desc, "impl": "FP64 oracle restating PDSolver_MG::Step",
                                     "ran_on": f"host cores only, one process (rank 0 of {args.gpus} requested)"},
                          "impl": "reference",
                          "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port",
                                           "sample": f"{args.steps} frames after {args.warmup} warm-up frames"},
                          "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    meshes, params, fixeds, tool, desc, mats = make_workload(args.workload, mg)
    os_ = make_oracles(meshes, params, fixeds, mats)
    oracle_frames(os_, tool, 0, args.warmup)
    t0 = time.perf_counter()
    oracle_frames(os_, tool, args.warmup, args.steps)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "impl": "FP64 oracle restating the configured PD multigrid frame",
                       "ran_on": f"host cores only, one process (rank 0 of {args.gpus} requested)"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} frames of the workload after {args.warmup} warm-up frames"},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# Learned smoother: training from the plain solver, accuracy check
# ---------------------------------------------------------------------------
LEARNED = ("beam", "blob")


TRAIN_RUNS = {"beam": (8, 10), "blob": (32, 20)}   # seeded runs, pairs every k frames (40 frames per run)


VALIDATION_FRAMES = 120   # held-out frames (into deep contact) that choose among the trained candidates


def train_network(mg, name, device, stream_ptr, runs=None, frames=40, every=None, sweeps=3, steps=20000,
                  candidates=4):
    """Pairs from the plain FP32 multigrid solver on seeded runs of the same scene (tool seeds other than
    the benchmark's), then the library's own trainer (Adam, 4096-pair minibatches) on `candidates`
    initialisations; the one whose learned V-cycles contract best on a held-out run is kept.  The blob
    (config 4) takes the configured 32 runs (~1M pairs); the beam headline 8 runs."""
    default_runs, default_every = TRAIN_RUNS.get(name, (8, 10))
    runs, every = runs or default_runs, every or default_every
    from multigridsoftbody_b200.learned import MLP, blob_scene, blob_tool_path
    t0 = time.perf_counter()
    if name == "blob":
        m, fixed, p = blob_scene()
        paths = [blob_tool_path(frames, seed=100 + r) for r in range(runs)]
    else:
        m = mg.box_mesh(12, 120, 12)
        fixed = (np.abs(m.positions[:, 1] - 10.0) < 1e-5).astype(np.uint8)
        p = mg.default_params(mg.SOLVER_MULTIGRID, levels=4, iterations=10, gravity=(0.0, 0.0, 0.0))
        paths = [capsule_path(frames, start=(0.0, 0.0, 1.5), seed=200 + r) for r in range(runs)]
    p.device = device
    p.stream = stream_ptr
    xs, ts = [], []
    for path in paths:
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        for f, (a, b) in enumerate(path):
            s.set_capsule(a, b, 0.3)
            s.step()
            if f % every == every - 1:
                x, t = s.smoother_pairs(sweeps)
                xs.append(x)
                ts.append(t)
        s.close()
    x, t = np.concatenate(xs), np.concatenate(ts)
    t1 = time.perf_counter()
    # candidates from different initialisations and minibatch orders, kept by how well their learned
    # V-cycles contract on a held-out run (tool seed 300, the learned form 1+1 sweeps, 2 passes)
    from multigridsoftbody_b200 import sweeps as swp
    from multigridsoftbody_b200.learned import held_out_contraction
    pv = swp.variant_params(p, (1, 1), 2, True)
    if name == "blob":
        val_path = blob_tool_path(VALIDATION_FRAMES, seed=300)
    else:
        val_path = capsule_path(VALIDATION_FRAMES, start=(0.0, 0.0, 1.5), seed=300)
    best, cands = None, []
    for k in range(candidates):
        net = MLP(device=device, seed=k)
        losses = net.train(x, t, steps=steps, batch=4096, lr=2e-3, seed=1 + k)
        score = held_out_contraction(net, m, fixed, pv, val_path)
        score.update(seed=k, loss_last=float(losses[-200:].mean()))
        cands.append(score)
        key = (score["failed_checks"], score["ratio_p99"])
        if best is None or key < best[0]:
            best = (key, net, losses, k)
    _, net, losses, kbest = best
    t2 = time.perf_counter()
    info = {"pairs": int(x.shape[0]), "runs": runs, "frames_per_run": frames, "distilled_jacobi_sweeps": sweeps,
            "train_steps": steps, "batch": 4096, "pair_generation_s": round(t1 - t0, 2),
            "train_and_select_s": round(t2 - t1, 2), "loss_first": float(losses[:20].mean()),
            "loss_last": float(losses[-200:].mean()), "candidates": cands, "chosen_seed": kbest,
            "selection": f"fewest failed checks, then the lowest 99th percentile of |r_after|/|r_before| per learned "
                         f"V-cycle, over {VALIDATION_FRAMES} frames of a held-out tool path (seed 300)"}
    return net, info


def accuracy(mg, meshes, fixeds, params, paths, net, variants, frames=100):
    """Max vertex error (largest Euclidean distance of a vertex) / bbox diagonal after `frames` frames
    from rest against the converged solver (mixed precision with 6 FP64-residual V-cycles per PD
    iteration, plain smoother), on each of `paths` ((label, tool) pairs), for each (sweeps, passes,
    learned) variant; err_over_diag is the worst over the paths."""
    from multigridsoftbody_b200 import sweeps as sw
    m, fixed = meshes[0], fixeds[0]
    refs = [sw.converged_positions(m, fixed, params[0], tool, frames) for _, tool in paths]
    diag = m.bbox_diagonal()
    out = {"frames": frames, "paths": [label + ", tool seed 1" for label, _ in paths],
           "error": "max over vertices of the Euclidean distance / bbox diagonal, worst over the paths",
           "reference": "GPU mixed precision, 6 V-cycles (FP64 residual) per PD iteration, plain smoother; "
                        "its distance from the FP64 oracle (6 V-cycles) over the same 100 frames is checked by "
                        "tests/test_gpu_headline.py"}
    for sweeps, passes, learned in variants:
        key = sw.variant_key(sweeps, passes, learned)
        if key in out:
            continue
        p = sw.variant_params(params[0], sweeps, passes, learned)
        errs, stats = [], [0, 0]
        for (label, tool), ref in zip(paths, refs):
            x, st = sw.run_positions(m, fixed, p, net if learned else None, tool, frames)
            errs.append(sw.max_vertex_error(x, ref) / diag)
            if st:
                stats = [stats[0] + st[0], stats[1] + st[1]]
        out[key] = {"err_over_diag": max(errs), "err_per_path": errs}
        if learned:
            out[key]["learned_vcycles"], out[key]["failed_checks"] = stats
    return out


# ---------------------------------------------------------------------------
# Sweep counts picked by accuracy (multigridsoftbody_b200.sweeps), the same search for both families
# ---------------------------------------------------------------------------
ERROR_BAR = 1e-5   # max vertex error / bbox diagonal after 100 frames
# The selection chooses among forms within half the bar on its held-out paths: a form just under the
# bar there (the learned 1-pass form: 8e-6) can be well over it on the check paths (2e-4 seen).
SELECTION_MARGIN = 0.5


def accuracy_paths(name, seed):
    """The tool paths the error bar is checked on, 100 frames each from rest: for the beam the config-1
    path as configured (capsule from z = 3, in contact from frame ~85) and the same motion started at
    z = 1.5 (in contact from frame ~10, deep in contact by frame 100: the stricter of the two); for the
    blob its tool path.  The selection uses seed 301, the check of the timed solver seed 1 (the timed
    frames run the z = 1.5 path with seed 1)."""
    from multigridsoftbody_b200.learned import blob_tool_path
    if name == "blob":
        paths = [("blob tool path", blob_tool_path(128, seed=seed))]
    else:
        paths = [("config-1 path from z=3", capsule_path(128, start=(0.0, 0.0, 3.0), seed=seed)),
                 ("in contact from z=1.5", capsule_path(128, start=(0.0, 0.0, 1.5), seed=seed))]

    def make(path):
        def tool(f):
            a, b = path[f % len(path)]
            return a[None], b[None], np.array([0.3], np.float32)
        return tool

    return [(label, make(p)) for label, p in paths]


# ---------------------------------------------------------------------------
# The reference's two-level schedule (PDSolver_MG) on the config-1 beam
# ---------------------------------------------------------------------------
def twolevel_scene(mg):
    """Fine: the 12x120x12-hex beam (103,680 tets); coarse: the same box at 4x40x4 hexes (3,840 tets),
    as the reference pairs cube120_12_12 with 40_4_4; top faces fixed; a sphere (r 0.8) swept along -x
    through the beam; reference constants (20 Jacobi/Chebyshev iterations per level)."""
    lo, hi = (-1.0, -10.0, -1.0), (1.0, 10.0, 1.0)
    fine = mg.box_mesh(12, 120, 12, lo, hi)
    coarse = mg.box_mesh(4, 40, 4, lo, hi)
    ff = (np.abs(fine.positions[:, 1] - hi[1]) < 1e-5).astype(np.uint8)
    cf = (np.abs(coarse.positions[:, 1] - hi[1]) < 1e-5).astype(np.uint8)
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)

    def sphere(f):
        return np.array([[1.5 - 0.01 * (f % 300), -3.0, 0.2]], np.float32), np.array([0.8], np.float32)

    desc = ("two-level schedule of the reference (PDSolver_MG): fine beam 12x120x12 hexes (20,449 verts, 103,680 "
            "tets), coarse 4x40x4 (3,840 tets), 20 Jacobi/Chebyshev iterations per level, sphere r 0.8 swept -x")
    return coarse, fine, cf, ff, p, sphere, desc


def run_twolevel(args):
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
    coarse, fine, cf, ff, p, sphere, desc = twolevel_scene(mg)
    p.device = local
    p.stream = stream.cuda_stream
    t = mg.TwoLevel(coarse, fine, p)
    t.set_fixed(cf, ff)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    with torch.cuda.stream(stream):
        for f in range(args.warmup):
            t.set_spheres(*sphere(f))
            t.step()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                evs[k][0].record(stream)
                t.set_spheres(*sphere(args.warmup + k))
                t.step()
                evs[k][1].record(stream)
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        e2e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            e2e[k][0].record(stream)
            t.set_spheres(*sphere(args.warmup + args.steps + k))
            t.step()
            t.positions(0)
            e2e[k][1].record(stream)
        torch.cuda.synchronize()
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e)
    from multigridsoftbody_b200.replicas import job_throughput, max_over_ranks
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], dist)
    if rank == 0:
        it = p.iterations
        launches = 2 + 3 * it + 1 + 2 * it + 1 + 1 + 2
        cpu = None
        if world == 1 and not args.no_cpu:
            from oracle.binding import OracleTwoLevel
            o = OracleTwoLevel(coarse, fine, p)
            o.set_fixed(cf, ff)
            o.set_spheres(*sphere(0))
            o.step()
            t0 = time.perf_counter()
            nfr = 0
            while nfr < args.cpu_frames and (nfr < 3 or time.perf_counter() - t0 < args.cpu_seconds):
                o.set_spheres(*sphere(1 + nfr))
                o.step()
                nfr += 1
            dt = time.perf_counter() - t0
            cpu = {"value": nfr / dt, "unit": "frames/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{nfr} frames of the same workload, FP64 oracle of the two-level schedule ({dt:.1f} s)"}
        line = {"metric": METRIC, "value": job_throughput(args.steps, world, ms), "unit": "frames/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": desc, "parallelism": f"replicas x{world}",
                           "l2": "flushed (256 MB write) before every timed frame, outside the timed span"},
                "clocks": clk.summary(),
                "e2e": {"value": job_throughput(args.steps, world, e2e_ms), "unit": "frames/s",
                        "h2d_bytes_per_step": 2 * (88 + 164), "d2h_bytes_per_step": fine.num_verts * 16},
                "gpu_launches": launches * args.steps, "roofline": None, "cpu_baseline": cpu}
        print(json.dumps(line))
    t.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import multigridsoftbody_b200 as mg
    from multigridsoftbody_b200 import sweeps as swp

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
    job_verts = sum(m.num_verts for m in meshes)
    job_bodies = len(meshes)
    meshes, params, fixeds, tool, mats, shard = shard_workload(meshes, params, fixeds, tool, mats, world, rank)
    for p in params:
        p.device = local
        p.stream = stream.cuda_stream
    net, net_info = None, None
    if args.workload in LEARNED and args.load_weights:
        from multigridsoftbody_b200.learned import MLP
        net = MLP(device=local, seed=0)
        net.params = np.load(args.load_weights)
        net_info = {"weights": os.path.basename(args.load_weights), "trained": "earlier run (--save-weights)"}
    elif args.workload in LEARNED:
        net, net_info = train_network(mg, args.workload, local, stream.cuda_stream,
                                      runs=args.train_runs or None, every=args.train_every or None)
        if args.save_weights and rank == 0:
            np.save(args.save_weights, net.params)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")   # 256 MB > L2

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    def shape(sv):
        """The coarse shape: --coarse-shape as given, else the autotuner's (none with --no-tune)."""
        if args.coarse_shape:
            split, _, dense = args.coarse_shape.partition(",")
            sv.set_coarse_split(int(split))
            sv.set_coarse_dense(dense == "dense")
            return {"split": sv.coarse_split(), "dense_operator": sv.coarse_dense(), "source": "--coarse-shape"}
        return sv.autotune(frames=5) if not args.no_tune else None

    def time_config(p, netx, tool_t, frames=60, warm=10):
        """ms per frame of one solver configuration: autotuned shape, L2 flushed before every frame."""
        sv = mg.Solver(meshes, [p])
        sv.set_fixed(fixeds[0])
        if netx is not None:
            sv.set_learned_smoother(netx, 0.5)
        shape(sv)
        with torch.cuda.stream(stream):
            for f in range(warm):
                apply_tool(sv, tool_t(f))
                sv.step()
            sv.synchronize()
            tev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
            for k in range(frames):
                flush.zero_()
                tev[k][0].record(stream)
                apply_tool(sv, tool_t(warm + k))
                sv.step()
                tev[k][1].record(stream)
            sv.synchronize()
        sv.close()
        return sum(a.elapsed_time(b) for a, b in tev) / frames

    # sweep counts of the learned solver: picked by accuracy on a held-out tool path (the plain
    # solver gets the same search for the comparison), or given, or the workload's
    selection, sweeps_source = None, "workload default"
    workload_params = [type(p).from_buffer_copy(p) for p in params]   # the CPU baseline runs these
    if args.sweeps:
        pre, post = (int(v) for v in args.sweeps.split(","))
        for p in params:
            p.pre_sweeps, p.post_sweeps = pre, post
            if args.passes:
                p.refinement_passes = args.passes
        sweeps_source = "--sweeps"
    elif net is not None and not args.no_compare and len(meshes) == 1:
        held = accuracy_paths(args.workload, 301)
        selection = swp.select_sweeps(meshes[0], fixeds[0], params[0], net, [t for _, t in held],
                                      time_fn=lambda p, netx: time_config(p, netx, held[-1][1]),
                                      bar=ERROR_BAR, time_all=True, margin=SELECTION_MARGIN)
        selection["held_out_paths"] = [label + ", tool seed 301" for label, _ in held]
        choice = selection["learned_mixed"]["chosen"]
        source = "selected by accuracy on held-out tool paths"
        if choice is None and selection["learned_mixed"]["candidates"]:
            # no learned form within the selection's margin: the most accurate one, not the default
            choice = min(selection["learned_mixed"]["candidates"], key=lambda r: r["err_over_diag"])
            source = "no learned form within the selection margin on the held-out paths: the most accurate one"
        if dist is not None:   # every rank runs rank 0's choice
            box = [choice, source]
            dist.broadcast_object_list(box, src=0)
            choice, source = box
        if choice is not None:
            params[0].pre_sweeps, params[0].post_sweeps = choice["sweeps"]
            params[0].refinement_passes = choice["passes"]
            sweeps_source = source
    solver = mg.Solver(meshes, params)
    for b, fx in enumerate(fixeds):
        solver.set_fixed(fx, body=b)
        if mats is not None:
            solver.set_material(*mats[b], body=b)
    if net is not None:
        solver.set_learned_smoother(net, 0.5)
    if args.broad_phase:
        solver.set_broad_phase(True)

    frame = 0
    tuned = shape(solver)
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
            pos_view, flag_view = solver.frame_view()   # positions (xyz) + contact flags, one readback, no copy
            e2e_evs[k][1].record(stream)
            frame += 1
        torch.cuda.synchronize()
        e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_evs)
        # live per-kernel profile of one frame (eager, events around every launch), cold L2
        flush.zero_()
        torch.cuda.synchronize()
        apply_tool(solver, tool(frame))
        prof = solver.profile_frame()
        frame += 1
        # kernel-only device time per launch: every launch of a kernel repeated back to back
        # inside the frame's own chain (no event nodes between them); the state is restored
        replay = {}
        for kname in ([] if args.no_replay else prof):
            if kname.startswith("k_bp_"):
                continue
            try:
                us, cnt = solver.time_kernel(kname, 20)
            except mg.MgsbError:
                continue
            replay[kname] = (us, cnt)
        # the plain FP32 multigrid, timed the same way: the configured form (1 V-cycle, 2+2 sweeps)
        # and every form that met the error bar in the selection
        plain_ms, plain_forms = {}, {}
        if net is not None and not args.no_compare:
            forms = [((2, 2), 1)]
            if selection:
                forms += [(tuple(r["sweeps"]), r["passes"]) for r in selection["plain_fp32"]["candidates"]
                          if "ms_per_frame" in r]
            if dist is not None:   # every rank times rank 0's list
                box = [forms]
                dist.broadcast_object_list(box, src=0)
                forms = box[0]
            for sweeps, passes in forms:
                plain_forms.setdefault(swp.variant_key(sweeps, passes, False), (tuple(sweeps), passes))
            for key, (sweeps, passes) in plain_forms.items():
                pp = swp.variant_params(params[0], sweeps, passes, False)
                sv = mg.Solver(meshes, [pp])
                sv.set_fixed(fixeds[0])
                shape(sv)
                for f in range(args.warmup):
                    apply_tool(sv, tool(f))
                    sv.step()
                sv.synchronize()
                barrier()
                pevs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                        for _ in range(args.steps)]
                for k in range(args.steps):
                    flush.zero_()
                    pevs[k][0].record(stream)
                    apply_tool(sv, tool(args.warmup + k))
                    sv.step()
                    pevs[k][1].record(stream)
                sv.synchronize()
                barrier()
                plain_ms[key] = sum(a.elapsed_time(b) for a, b in pevs)
                sv.close()
    from multigridsoftbody_b200.replicas import job_throughput, max_over_ranks, sharded_throughput
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], dist)
    if shard is not None:   # a frame advances every body of the batch once, on the rank that holds it
        def job_throughput(frames, _world, max_ms):
            return sharded_throughput(frames, max_ms)
    comparison = None
    if net is not None and not args.no_compare:
        keys = list(plain_ms)
        times = max_over_ranks([plain_ms[k] for k in keys], dist)
        learned_key = swp.variant_key((params[0].pre_sweeps, params[0].post_sweeps), params[0].refinement_passes,
                                         True)
        comparison = {"learned": learned_key, "sweeps_source": sweeps_source, "network": net_info,
                      "error_bar_over_diag": ERROR_BAR, "selection": selection}
        for k, t in zip(keys, times):
            comparison[k] = {"frames_per_s": job_throughput(args.steps, world, t), "ms_per_step": t / args.steps,
                             "ratio": job_throughput(args.steps, world, ms) / job_throughput(args.steps, world, t)}
        if rank == 0 and world == 1:
            variants = [((params[0].pre_sweeps, params[0].post_sweeps), params[0].refinement_passes, True)]
            variants += [(sw, ps, False) for sw, ps in plain_forms.values()]
            acc = accuracy(mg, meshes, fixeds, params, accuracy_paths(args.workload, 1), net, variants)
            comparison["accuracy"] = acc
            comparison["learned_meets_bar"] = acc[learned_key]["err_over_diag"] <= ERROR_BAR
            # the headline ratio: against the fastest timed plain FP32 form that meets the bar on this path
            at_bar = [k for k in keys if acc[k]["err_over_diag"] <= ERROR_BAR]
            if at_bar:
                best = min(at_bar, key=lambda k: comparison[k]["ms_per_step"])
                comparison["plain_fp32_at_bar"] = best
                comparison["ratio_vs_plain_fp32_at_bar"] = comparison[best]["ratio"]
            # equal error in the strict sense: the fastest plain form at most as far from the converged
            # frame as the learned solver (matters where every form is far inside the bar, e.g. the blob)
            le = acc[learned_key]["err_over_diag"]
            at_err = [k for k in keys if acc[k]["err_over_diag"] <= le]
            comparison["plain_fp32_at_learned_error"] = (min(at_err, key=lambda k: comparison[k]["ms_per_step"])
                                                         if at_err else None)
            comparison["ratio_vs_plain_fp32_at_learned_error"] = (
                comparison[comparison["plain_fp32_at_learned_error"]]["ratio"] if at_err else None)
    value = job_throughput(args.steps, world, ms)
    e2e_value = job_throughput(args.steps, world, e2e_ms)
    if rank == 0:
        launches = solver.launches_per_frame()
        if net is not None and comparison is not None:
            # every learned V-cycle this solver ran (warm-up, timed, e2e, profiled and replayed frames):
            # checks, and checks failed (a frame with a failed check was recomputed with plain V-cycles)
            comparison["learned_checks_this_solver"] = list(solver.learned_stats())
        # the dominant kernel by its kernel-only time per frame, among those with an algorithmic-byte figure
        top_any = None
        if replay:
            top_any = max(replay, key=lambda k: replay[k][0] * replay[k][1])
            with_figure = {k: v for k, v in replay.items() if algorithmic_bytes(k, solver, meshes, params[0]) is not None}
            replay_f = with_figure or replay
            kname = max(replay_f, key=lambda k: replay_f[k][0] * replay_f[k][1])
            kavg_ms = replay[kname][0] / 1e3
            share = replay[kname][0] * replay[kname][1] / sum(u * c for u, c in replay.values())
            source = "replay: each launch repeated 20x back to back in the frame's chain, CUDA events"
        else:
            kname = max(prof, key=lambda k: prof[k][0])
            kavg_ms = prof[kname][0] / max(prof[kname][1], 1)
            share = prof[kname][0] / sum(v[0] for v in prof.values())
            source = "profiled frame: CUDA event nodes around every launch"
        alg = algorithmic_bytes(kname, solver, meshes, params[0])
        peak, peak_kind = measured_peaks()
        roof = None
        if alg is not None:
            ach = alg / (kavg_ms / 1e3) / 1e9
            roof = {"bound": "hbm", "kernel": kname, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "traffic": ncu_traffic(kname, args.workload), "peak_kind": peak_kind,
                    "algorithmic_bytes_per_launch": alg, "avg_launch_ms": kavg_ms,
                    "duration_source": source, "share_of_frame": share,
                    "avg_launch_ms_profiled": prof[kname][0] / max(prof[kname][1], 1)}
            if top_any is not None and top_any != kname:
                roof["dominant_kernel_without_a_figure"] = top_any
            # whole frame: every launch of every kernel with an algorithmic-byte figure, over the frame time
            fb, missing = 0.0, []
            for k, (kms, cnt) in prof.items():
                b = algorithmic_bytes(k, solver, meshes, params[0])
                if b is None:
                    missing.append(k)
                else:
                    fb += b * cnt
            fms = ms / args.steps
            roof["frame"] = {"algorithmic_bytes": fb, "ms": fms, "achieved_gbs": fb / (fms / 1e3) / 1e9,
                             "frame_frac": fb / (fms / 1e3) / 1e9 / peak,
                             "survey_estimate_bytes": params[0].iterations * (
                                 168.0 * sum(m.num_tets for m in meshes) + 1139.0 * sum(m.num_verts for m in meshes)),
                             "kernels_without_a_figure": sorted(missing)}
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_baseline(meshes, workload_params, fixeds, tool, mats, args,
                               comparison.get("plain_fp32_at_bar") if comparison else None)
        # whole job: body table (88 B per body) + sphere set per rank; packed xyz positions + contact
        # flags (16 B per vertex) + the non-finite flag per rank
        h2d = job_bodies * 88 + 164 * world if shard is not None else (len(meshes) * 88 + 164) * world
        d2h = (job_verts * 16 + 4 * world) if shard is not None else (nverts * 16 + 4) * world
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if shard is not None else "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": desc,
                           "variant": ("learned smoother + " if net is not None else "")
                           + ("mixed precision multigrid" if params[0].precision == 1 else "plain FP32 multigrid"),
                           "parallelism": (f"bodies sharded over {world} ranks (rank 0: {len(meshes)} of "
                                           f"{job_bodies} bodies), no data-path collective"
                                           if shard is not None else f"replicas x{world}"),
                           "l2": "flushed (256 MB write) before every timed frame, outside the timed span",
                           "autotuned_coarse_kernel": tuned,
                           "contact_broad_phase": "uniform grid" if args.broad_phase else "all surface vertices",
                           "sweeps_per_level": [params[0].pre_sweeps, params[0].post_sweeps],
                           "refinement_passes": params[0].refinement_passes, "sweeps_source": sweeps_source},
                "clocks": clk.summary(),
                "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches * args.steps,
                "roofline": roof,
                "cpu_baseline": cpu,
                "comparison": comparison,
                "kernels": {k: {"ms_per_frame": v[0], "launches": v[1],
                                "replay_us_per_launch": replay[k][0] if k in replay else None}
                            for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}}
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
    ap.add_argument("--sweeps", default=None,
                    help="PRE,POST sweeps per level (default: picked by accuracy for the learned workloads)")
    ap.add_argument("--passes", type=int, default=0,
                    help="V-cycles per PD iteration with --sweeps (default: the workload's)")
    ap.add_argument("--no-replay", action="store_true",
                    help="roofline from the profiled frame only (no kernel replay frames: short ncu launch lists)")
    ap.add_argument("--cpu-frames", type=int, default=1000, help="most frames of the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="the CPU baseline runs frames until this much time has passed (at least 3 frames)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--coarse-shape", default="",
                    help="SPLIT or SPLIT,dense: fixed coarse split (and dense coarse operator) instead of autotuning")
    ap.add_argument("--broad-phase", action="store_true", help="uniform-grid broad phase for the tool contact")
    ap.add_argument("--no-compare", action="store_true",
                    help="learned workloads: skip the plain-solver timings and the accuracy runs (profiling)")
    ap.add_argument("--train-runs", type=int, default=0, help="learned workloads: seeded training runs (0: workload's)")
    ap.add_argument("--train-every", type=int, default=0, help="learned workloads: pairs every k frames (0: workload's)")
    ap.add_argument("--save-weights", default="", help="learned workloads: save the trained network (.npy)")
    ap.add_argument("--load-weights", default="", help="learned workloads: use these weights instead of training")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        # no launcher: start one process per GPU here (rendezvous on 127.0.0.1)
        import socket
        import torch.multiprocessing as tmp
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
        sk.close()
        tmp.spawn(_rank_main, args=(args, port), nprocs=args.gpus, join=True)
        return
    dispatch(args)


def dispatch(args):
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "twolevel":
        run_twolevel(args)
    else:
        run_ours(args)


def _rank_main(rank, args, port):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(args.gpus),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dispatch(args)


if __name__ == "__main__":
    main()
