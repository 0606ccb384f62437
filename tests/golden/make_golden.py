"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference (buuugyellow/MultiGridSoftBody) is compiled headless by
oracle/ref_build.sh into oracle/_ref/libmgsb_ref.so; this script calls it:

    python tests/golden/make_golden.py cpu     # precompute, polar, mesh I/O (no GPU)
    python tests/golden/make_golden.py gpu     # PDSolver::Step trajectories (needs a GPU)
    python tests/golden/make_golden.py gpu_mg2 # PDSolver_MG::Step trajectories (needs a GPU)

Inputs are generated here (seeded); no reference data file is copied.
Outputs: ref_cpu.npz, ref_traj.npz, ref_mg2_traj.npz (small, committed).

beam_smoother.npy in this folder is not from the reference: it is the
headline's learned-smoother network (4,995 float32 parameters), trained on a
B200 by the library's own trainer and written by

    python bench.py --steps 50 --warmup 5 --no-cpu --save-weights tests/golden/beam_smoother.npy

The profiling commands in profiles/ load it (--load-weights) so that a
profiled frame needs no training run.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libmgsb_ref.so")

# Golden scene of the trajectory fixture: 4x14x4 hexes (1,344 tets, a multiple
# of 56 so the reference's 504-thread local-step blocks are always full),
# top face fixed, a sphere pushed through the beam.
TRAJ_DIMS = (4, 14, 4)
TRAJ_LO = (-1.0, -7.0, -1.0)
TRAJ_HI = (1.0, 7.0, 1.0)
TRAJ_FRAMES = 100
TRAJ_ITERS = 20
TRAJ_KEEP = list(range(9, TRAJ_FRAMES, 10))


def traj_sphere_path(frames: int = TRAJ_FRAMES) -> np.ndarray:
    """Per frame (cx, cy, cz, r): radius 0.8, moving -x by 0.05 per frame."""
    path = np.zeros((frames, 4), np.float32)
    for f in range(frames):
        path[f] = (2.5 - 0.05 * f, -3.0, 0.2, 0.8)
    return path


def _lib():
    if not os.path.exists(REF_LIB):
        raise SystemExit(f"{REF_LIB} missing: run oracle/ref_build.sh first")
    lib = C.CDLL(REF_LIB)
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int32)
    lib.ref_precompute.argtypes = [fp, C.c_int, ip, C.c_int, C.c_float, fp, fp, fp, fp, fp]
    lib.ref_rotation.argtypes = [fp, fp, fp]
    lib.ref_inverse3.argtypes = [fp, fp]
    lib.ref_inverse3.restype = C.c_float
    lib.ref_barycentric.argtypes = [fp, fp, fp, fp, fp, fp]
    lib.ref_read_msh.argtypes = [C.c_char_p, ip, ip, ip]
    lib.ref_read_msh_arrays.argtypes = [fp, ip, ip, ip]
    lib.ref_extract_surface.argtypes = [fp, C.c_int, ip, C.c_int, ip, ip, C.c_int]
    lib.ref_extract_surface.restype = C.c_int
    lib.ref_run.argtypes = [fp, C.c_int, ip, C.c_int, C.POINTER(C.c_uint8), C.c_int, C.c_int, fp, fp, ip, fp]
    lib.ref_run.restype = C.c_int
    u8 = C.POINTER(C.c_uint8)
    lib.ref_mg2_run.argtypes = [fp, C.c_int, ip, C.c_int, fp, C.c_int, ip, C.c_int, u8, u8, C.c_int, fp, fp, fp, fp]
    lib.ref_mg2_run.restype = C.c_int
    return lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def write_msh(path: str, pos: np.ndarray, tets: np.ndarray) -> None:
    """gmsh 2.2 ASCII writer (nodes + tets, two tags per element)."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(pos))
        for i, p in enumerate(pos):
            f.write("%d %.9g %.9g %.9g\n" % (i + 1, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % len(tets))
        for e, t in enumerate(tets):
            f.write("%d 4 2 0 1 %d %d %d %d\n" % (e + 1, t[0] + 1, t[1] + 1, t[2] + 1, t[3] + 1))
        f.write("$EndElements\n")


def jittered_box(nx, ny, nz, seed):
    import multigridsoftbody_b200 as mg
    m = mg.box_mesh(nx, ny, nz, (-1, -3, -1), (1, 3, 1))
    rng = np.random.default_rng(seed)
    h = min(2.0 / nx, 6.0 / ny, 2.0 / nz)
    pos = m.positions + rng.uniform(-0.15 * h, 0.15 * h, m.positions.shape).astype(np.float32)
    return pos.astype(np.float32), m.tets.astype(np.int32)


def make_cpu() -> None:
    lib = _lib()
    out = {}
    # --- precompute (PDSolver::InitVolumeConstraint) on a jittered box
    pos, tets = jittered_box(2, 6, 2, seed=5)
    V, T = len(pos), len(tets)
    inv = np.zeros(9 * T, np.float32)
    ac = np.zeros(12 * T, np.float32)
    vol = np.zeros(T, np.float32)
    mass = np.zeros(V, np.float32)
    diag = np.zeros(V, np.float32)
    lib.ref_precompute(_f(pos), V, _i(tets), T, 8000.0, _f(inv), _f(ac), _f(vol), _f(mass), _f(diag))
    out.update(pre_pos=pos, pre_tets=tets, pre_inv=inv.reshape(T, 9), pre_ac=ac.reshape(T, 12), pre_vol=vol,
               pre_mass=mass, pre_diag=diag)
    # --- polar decomposition (GetRotation_D) on seeded matrices
    rng = np.random.default_rng(11)
    Fs = []
    for k in range(300):
        if k < 200:
            F = np.eye(3) + rng.normal(0, 0.25, (3, 3))          # moderate deformation
        elif k < 250:
            Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Q *= np.sign(np.linalg.det(Q))
            F = Q @ np.diag(rng.uniform(0.3, 2.0, 3))            # rotation x stretch
        else:
            F = np.eye(3) + rng.normal(0, 0.05, (3, 3))          # near identity
        if np.linalg.det(F) <= 0.05:
            F[:, 0] *= -1
        Fs.append(F.astype(np.float32))
    Fs = np.stack(Fs)
    Rs = np.zeros_like(Fs)
    for k in range(len(Fs)):
        R = np.zeros(9, np.float32)
        d = C.c_float()
        lib.ref_rotation(_f(np.ascontiguousarray(Fs[k].reshape(9))), _f(R), C.byref(d))
        Rs[k] = R.reshape(3, 3)
    out.update(rot_F=Fs, rot_R=Rs)
    # --- 3x3 inverse (Matrix_Inverse_3)
    A = (np.eye(3) + rng.normal(0, 0.3, (64, 3, 3))).astype(np.float32)
    Ai = np.zeros_like(A)
    dets = np.zeros(64, np.float32)
    for k in range(64):
        R = np.zeros(9, np.float32)
        dets[k] = lib.ref_inverse3(_f(np.ascontiguousarray(A[k].reshape(9))), _f(R))
        Ai[k] = R.reshape(3, 3)
    out.update(inv_A=A, inv_R=Ai, inv_det=dets)
    # --- msh reader + boundary-face extraction on a generated mesh file
    mpos, mtets = jittered_box(3, 5, 2, seed=9)
    tmp = os.path.join(HERE, "_tmp_golden.msh")
    write_msh(tmp, mpos, mtets)
    nv, nt, nf = C.c_int(), C.c_int(), C.c_int()
    lib.ref_read_msh(tmp.encode(), C.byref(nv), C.byref(nt), C.byref(nf))
    rp = np.zeros(3 * nv.value, np.float32)
    rt = np.zeros(4 * nt.value, np.int32)
    rf = np.zeros(3 * nf.value, np.int32)
    ro = np.zeros(nf.value, np.int32)
    lib.ref_read_msh_arrays(_f(rp), _i(rt), _i(rf), _i(ro))
    with open(tmp) as fh:
        msh_text = fh.read()
    os.remove(tmp)
    out.update(msh_text=np.frombuffer(msh_text.encode(), np.uint8), msh_pos=rp.reshape(-1, 3),
               msh_tets=rt.reshape(-1, 4), msh_tris=rf.reshape(-1, 3), msh_opp=ro)
    # --- surface extraction on a plain box (4x40x4 -> 1,344 faces)
    import multigridsoftbody_b200 as mg
    b = mg.box_mesh(2, 8, 3)
    cap = 10000
    tris = np.zeros(3 * cap, np.int32)
    opp = np.zeros(cap, np.int32)
    F = lib.ref_extract_surface(_f(b.positions), b.num_verts, _i(b.tets), b.num_tets, _i(tris), _i(opp), cap)
    out.update(surf_tets=b.tets, surf_tris=tris[: 3 * F].reshape(-1, 3), surf_opp=opp[:F])
    # --- barycentric coordinates
    P = rng.uniform(-0.2, 1.2, (32, 3)).astype(np.float32)
    tet = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32) + rng.normal(0, 0.05, (4, 3)).astype(np.float32)
    W = np.zeros((32, 4), np.float32)
    for k in range(32):
        w = np.zeros(4, np.float32)
        lib.ref_barycentric(_f(P[k]), _f(tet[0]), _f(tet[1]), _f(tet[2]), _f(tet[3]), _f(w))
        W[k] = w
    out.update(bary_P=P, bary_tet=tet, bary_W=W)
    np.savez_compressed(os.path.join(HERE, "ref_cpu.npz"), **out)
    print("wrote ref_cpu.npz", {k: v.shape for k, v in out.items()})


def traj_scene():
    import multigridsoftbody_b200 as mg
    m = mg.box_mesh(*TRAJ_DIMS, TRAJ_LO, TRAJ_HI)
    fixed = (np.abs(m.positions[:, 1] - TRAJ_HI[1]) < 1e-5).astype(np.uint8)
    return m, fixed


def make_gpu() -> None:
    lib = _lib()
    m, fixed = traj_scene()
    V, T = m.num_verts, m.num_tets
    assert T % 56 == 0
    path = traj_sphere_path()
    pos = np.zeros((TRAJ_FRAMES, V, 3), np.float32)
    flags = np.zeros((TRAJ_FRAMES, V), np.int32)
    ms = np.zeros(TRAJ_FRAMES, np.float32)
    st = lib.ref_run(_f(np.ascontiguousarray(m.positions)), V, _i(np.ascontiguousarray(m.tets)), T,
                     fixed.ctypes.data_as(C.POINTER(C.c_uint8)), TRAJ_ITERS, TRAJ_FRAMES, _f(path), _f(pos), _i(flags),
                     _f(ms))
    if st != 0:
        raise SystemExit(f"ref_run failed with status {st}")
    # a second identical run: the reference's float atomics make frames differ run to run
    pos2 = np.zeros_like(pos)
    st = lib.ref_run(_f(np.ascontiguousarray(m.positions)), V, _i(np.ascontiguousarray(m.tets)), T,
                     fixed.ctypes.data_as(C.POINTER(C.c_uint8)), TRAJ_ITERS, TRAJ_FRAMES, _f(path), _f(pos2), None,
                     None)
    if st != 0:
        raise SystemExit(f"ref_run (repeat) failed with status {st}")
    rerun = np.abs(pos - pos2).reshape(TRAJ_FRAMES, -1).max(1)
    out_dir = sys.argv[2] if len(sys.argv) > 2 else HERE
    np.savez_compressed(os.path.join(out_dir, "ref_traj.npz"), frames=np.array(TRAJ_KEEP), positions=pos[TRAJ_KEEP],
                        flags=flags[TRAJ_KEEP], ms=ms, rerun_maxdiff=rerun)
    print("run-to-run max difference of the reference:", float(rerun.max()))
    print("wrote ref_traj.npz; mean Step() ms", float(ms[5:].mean()))


# Two-level golden scene: the trajectory beam as the fine mesh and the same box
# with half the hexes per axis as the coarse mesh (nested: every fine vertex lies
# in a coarse tet and every coarse vertex is a fine vertex); top faces fixed.
MG2_COARSE_DIMS = (2, 7, 2)
MG2_FRAMES = 60
MG2_KEEP = list(range(9, MG2_FRAMES, 10))


def mg2_scene():
    import multigridsoftbody_b200 as mg
    fine = mg.box_mesh(*TRAJ_DIMS, TRAJ_LO, TRAJ_HI)
    coarse = mg.box_mesh(*MG2_COARSE_DIMS, TRAJ_LO, TRAJ_HI)
    ff = (np.abs(fine.positions[:, 1] - TRAJ_HI[1]) < 1e-5).astype(np.uint8)
    cf = (np.abs(coarse.positions[:, 1] - TRAJ_HI[1]) < 1e-5).astype(np.uint8)
    return coarse, fine, cf, ff


def make_gpu_mg2() -> None:
    lib = _lib()
    coarse, fine, cf, ff = mg2_scene()
    path = traj_sphere_path(MG2_FRAMES)
    runs = []
    for rep in range(2):
        fpos = np.zeros((MG2_FRAMES, fine.num_verts, 3), np.float32)
        cpos = np.zeros((MG2_FRAMES, coarse.num_verts, 3), np.float32)
        ms = np.zeros(MG2_FRAMES, np.float32)
        st = lib.ref_mg2_run(_f(np.ascontiguousarray(coarse.positions)), coarse.num_verts,
                             _i(np.ascontiguousarray(coarse.tets)), coarse.num_tets,
                             _f(np.ascontiguousarray(fine.positions)), fine.num_verts, _i(np.ascontiguousarray(fine.tets)),
                             fine.num_tets, cf.ctypes.data_as(C.POINTER(C.c_uint8)),
                             ff.ctypes.data_as(C.POINTER(C.c_uint8)), MG2_FRAMES, _f(path), _f(fpos), _f(cpos), _f(ms))
        if st != 0:
            raise SystemExit(f"ref_mg2_run failed with status {st}")
        runs.append((fpos, cpos, ms))
    rerun = np.abs(runs[0][0] - runs[1][0]).reshape(MG2_FRAMES, -1).max(1)
    out_dir = sys.argv[2] if len(sys.argv) > 2 else HERE
    np.savez_compressed(os.path.join(out_dir, "ref_mg2_traj.npz"), frames=np.array(MG2_KEEP),
                        fine=runs[0][0][MG2_KEEP], coarse=runs[0][1][MG2_KEEP], ms=runs[0][2], rerun_maxdiff=rerun)
    print("run-to-run max difference of the reference:", float(rerun.max()))
    print("wrote ref_mg2_traj.npz; mean Step() ms", float(runs[0][2][5:].mean()))


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "cpu"
    {"cpu": make_cpu, "gpu": make_gpu, "gpu_mg2": make_gpu_mg2}[what]()
