"""Time the reference's own GPU frame beside the build's reference kind on one GPU.

    python oracle/time_ref_gpu.py [--frames 60] [--warmup 10]

The reference (buuugyellow/MultiGridSoftBody) compiled headless by
oracle/ref_build.sh into oracle/_ref/libmgsb_ref.so runs PDSolver::Step
(PDSolver.cpp:243-293: 20 Jacobi/Chebyshev iterations, float atomics, its
render readback) through ref_run in oracle/ref_driver.cu; the build runs the
same frame as its MGSB_SOLVER_REFERENCE_JACOBI kind through the C ABI
(mgsb_step + mgsb_get_positions, the same readback).  Mesh: the box
[-1,1]x[-10,10]x[-1,1] as 12x112x12 hexes (19,097 vertices, 96,768 tets, a
multiple of 56, so every 504-thread block of the reference's getTetFRV2 is full
and no thread returns before its __syncthreads, PDSolverAc.cu:450,473), top
face fixed, a sphere of radius 0.8 swept along -x through the beam.  Both
times are wall-clock per frame with the frame's synchronisation inside (the
reference's Step synchronises itself).  Measurement infrastructure only; prints
one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
REF_LIB = os.path.join(HERE, "_ref", "libmgsb_ref.so")


def sphere_path(frames):
    """Per frame (cx, cy, cz, r)."""
    return np.array([(1.5 - 0.01 * f, -3.0, 0.2, 0.8) for f in range(frames)], np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--dims", default="12,112,12")
    args = ap.parse_args()
    import multigridsoftbody_b200 as mg

    nx, ny, nz = (int(v) for v in args.dims.split(","))
    m = mg.box_mesh(nx, ny, nz)
    fixed = (np.abs(m.positions[:, 1] - 10.0) < 1e-5).astype(np.uint8)
    V, T = m.num_verts, m.num_tets
    if T % 56:
        raise SystemExit(f"{T} tets is not a multiple of 56: the reference's local step would skip a barrier")
    total = args.warmup + args.frames
    path = sphere_path(total)
    out = {"mesh": f"box {nx}x{ny}x{nz} hexes ({V} verts, {T} tets)", "iterations": 20,
           "frames_timed": args.frames, "warmup": args.warmup}
    # the reference's own PDSolver::Step
    lib = C.CDLL(REF_LIB)
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
    lib.ref_run.argtypes = [fp, C.c_int, ip, C.c_int, C.POINTER(C.c_uint8), C.c_int, C.c_int, fp, fp, ip, fp]
    ms = np.zeros(total, np.float32)
    pos = np.ascontiguousarray(m.positions, np.float32)
    tets = np.ascontiguousarray(m.tets, np.int32)
    traj = np.zeros((total, V, 3), np.float32)
    st = lib.ref_run(pos.ctypes.data_as(fp), V, tets.ctypes.data_as(ip), T, fixed.ctypes.data_as(C.POINTER(C.c_uint8)),
                     20, total, path.ctypes.data_as(fp), traj.ctypes.data_as(fp), None, ms.ctypes.data_as(fp))
    if st != 0:
        raise SystemExit(f"ref_run failed with status {st}")
    ref_ms = float(ms[args.warmup:].mean())
    out["reference_step_ms"] = ref_ms
    # the build's reference kind, same frame, same readback
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    t_ours = []
    x = None
    for f in range(total):
        t0 = time.perf_counter()
        s.set_spheres(path[f:f + 1, :3], path[f:f + 1, 3])
        s.step()
        x = s.positions()
        t_ours.append(time.perf_counter() - t0)
    ours_ms = 1e3 * float(np.mean(t_ours[args.warmup:]))
    out["build_reference_kind_ms"] = ours_ms
    out["speedup"] = ref_ms / ours_ms
    out["max_vertex_distance_over_diag_last_frame"] = float(
        np.sqrt(((x - traj[-1]) ** 2).sum(1)).max() / m.bbox_diagonal())
    s.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
