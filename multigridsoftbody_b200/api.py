"""Python host API over the C ABI (include/mgsb.h): meshes, solvers, batches."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import MgsbError, Params


def _check(status: int, handle=None) -> None:
    if status != 0:
        msg = ""
        if handle:
            raw = L.load().mgsb_last_error_string(handle)
            msg = raw.decode() if raw else ""
        raise MgsbError(status, msg)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u8ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


# ---------------------------------------------------------------------------
# Meshes
# ---------------------------------------------------------------------------
@dataclass
class TetMesh:
    positions: np.ndarray            # (V, 3) float32
    tets: np.ndarray                 # (T, 4) int32
    grid_dims: tuple = (0, 0, 0)
    tris: np.ndarray | None = None   # (F, 3) boundary faces
    tri_opposite: np.ndarray | None = None

    @property
    def num_verts(self) -> int:
        return int(self.positions.shape[0])

    @property
    def num_tets(self) -> int:
        return int(self.tets.shape[0])

    def bbox_diagonal(self) -> float:
        return float(np.linalg.norm(self.positions.max(0).astype(np.float64) - self.positions.min(0)))

    def as_c(self) -> tuple[L.Mesh, tuple]:
        pos = np.ascontiguousarray(self.positions, dtype=np.float32)
        tets = np.ascontiguousarray(self.tets, dtype=np.int32)
        m = L.Mesh()
        m.num_verts = pos.shape[0]
        m.num_tets = tets.shape[0]
        m.positions = _fptr(pos)
        m.tets = _iptr(tets)
        for c in range(3):
            m.grid_dims[c] = int(self.grid_dims[c])
        return m, (pos, tets)   # keep the arrays alive with the struct


def _take_mesh(ptr) -> TetMesh:
    lib = L.load()
    d = ptr.contents
    V, T = d.num_verts, d.num_tets
    pos = np.ctypeslib.as_array(d.positions, shape=(V * 3,)).reshape(V, 3).copy()
    tets = np.ctypeslib.as_array(d.tets, shape=(T * 4,)).reshape(T, 4).copy()
    tris = opp = None
    if d.num_tris > 0:
        tris = np.ctypeslib.as_array(d.tris, shape=(d.num_tris * 3,)).reshape(-1, 3).copy()
        opp = np.ctypeslib.as_array(d.tri_opposite, shape=(d.num_tris,)).copy()
    dims = tuple(int(d.grid_dims[c]) for c in range(3))
    lib.mgsb_mesh_free(ptr)
    return TetMesh(pos, tets, dims, tris, opp)


def box_mesh(nx: int, ny: int, nz: int, lo=(-1.0, -10.0, -1.0), hi=(1.0, 10.0, 1.0)) -> TetMesh:
    """Box split into nx*ny*nz hexes, 6 Kuhn tets each."""
    lib = L.load()
    out = C.POINTER(L.MeshData)()
    lo_a = np.asarray(lo, dtype=np.float32)
    hi_a = np.asarray(hi, dtype=np.float32)
    _check(lib.mgsb_mesh_box(nx, ny, nz, _fptr(lo_a), _fptr(hi_a), C.byref(out)))
    return _take_mesh(out)


def blob_mesh(gx=64, gy=32, gz=48, spacing=0.25, semi_axes=(6.0, 3.0, 4.0), noise_amp=0.15, noise_period=2.0,
              seed=3) -> TetMesh:
    """Organ-like voxel blob (ellipsoid + seeded value noise), 6 Kuhn tets per voxel."""
    lib = L.load()
    out = C.POINTER(L.MeshData)()
    ax = np.asarray(semi_axes, dtype=np.float32)
    _check(lib.mgsb_mesh_blob(gx, gy, gz, spacing, _fptr(ax), noise_amp, noise_period, seed, C.byref(out)))
    return _take_mesh(out)


def read_msh(path: str) -> TetMesh:
    """gmsh 2.2 ASCII reader (tets only), like SoftObject::ReadFromFile."""
    lib = L.load()
    out = C.POINTER(L.MeshData)()
    _check(lib.mgsb_mesh_read_msh(path.encode(), C.byref(out)))
    return _take_mesh(out)


def extract_surface(mesh: TetMesh) -> TetMesh:
    """Fill mesh.tris / mesh.tri_opposite like SoftObject::TetFaceExtraction."""
    lib = L.load()
    d = L.MeshData()
    pos = np.ascontiguousarray(mesh.positions, dtype=np.float32)
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    d.num_verts, d.num_tets = pos.shape[0], tets.shape[0]
    # The library frees tris/opposite only; positions/tets stay owned by numpy.
    d.positions = _fptr(pos)
    d.tets = _iptr(tets)
    _check(lib.mgsb_mesh_extract_surface(C.byref(d)))
    F = d.num_tris
    tris = np.ctypeslib.as_array(d.tris, shape=(max(F, 1) * 3,))[: F * 3].reshape(-1, 3).copy()
    opp = np.ctypeslib.as_array(d.tri_opposite, shape=(max(F, 1),))[:F].copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(d.tris, C.c_void_p))
    libc.free(C.cast(d.tri_opposite, C.c_void_p))
    mesh.tris, mesh.tri_opposite = tris, opp
    return mesh


def value_noise(x: float, y: float, z: float, period: float, seed: int) -> float:
    return float(L.load().mgsb_value_noise(x, y, z, period, seed))


# ---------------------------------------------------------------------------
# Parameters
# ---------------------------------------------------------------------------
def default_params(kind: int = L.SOLVER_MULTIGRID, **overrides) -> Params:
    p = Params()
    _check(L.load().mgsb_default_params(kind, C.byref(p)))
    for k, v in overrides.items():
        if k == "gravity":
            for c in range(3):
                p.gravity[c] = float(v[c])
        else:
            setattr(p, k, v)
    return p


def params_dict(p: Params) -> dict:
    d = {}
    for name, _ in Params._fields_:
        v = getattr(p, name)
        d[name] = list(v) if name == "gravity" else v
    return d


# ---------------------------------------------------------------------------
# Solver handle
# ---------------------------------------------------------------------------
class Solver:
    """One handle holding one or more bodies (a batch)."""

    def __init__(self, meshes, params, _handle=None):
        self._lib = L.load()
        if isinstance(meshes, TetMesh):
            meshes = [meshes]
        if isinstance(params, Params):
            params = [params] * len(meshes)
        self.meshes = list(meshes)
        self.params = list(params)
        cm = (L.Mesh * len(meshes))()
        self._keep = []
        for i, m in enumerate(meshes):
            s, keep = m.as_c()
            cm[i] = s
            self._keep.append(keep)
        cp = (Params * len(params))(*params)
        h = C.c_void_p()
        if len(meshes) == 1:
            st = self._lib.mgsb_create(C.byref(cm[0]), C.byref(cp[0]), C.byref(h))
        else:
            st = self._lib.mgsb_batch_create(len(meshes), cm, cp, C.byref(h))
        if st != 0:
            raise MgsbError(st, "create failed")
        self.h = h
        self._keep = None

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "h", None):
            self._lib.mgsb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- sizes
    @property
    def num_bodies(self) -> int:
        n = C.c_int32()
        _check(self._lib.mgsb_num_bodies(self.h, C.byref(n)), self.h)
        return n.value

    def num_verts(self, body: int = 0) -> int:
        n = C.c_int32()
        _check(self._lib.mgsb_num_verts(self.h, body, C.byref(n)), self.h)
        return n.value

    def num_tets(self, body: int = 0) -> int:
        n = C.c_int32()
        _check(self._lib.mgsb_num_tets(self.h, body, C.byref(n)), self.h)
        return n.value

    # -- inputs
    def get_params(self) -> Params:
        """The parameters in force (mgsb_get_params)."""
        p = Params()
        _check(self._lib.mgsb_get_params(self.h, C.byref(p)), self.h)
        return p

    def set_params(self, params: Params = None, **changes) -> None:
        """Change parameters between frames (mgsb_set_params): a full Params, or keyword changes to the
        ones in force (gravity as a 3-sequence)."""
        p = Params.from_buffer_copy(params if params is not None else self.get_params())
        for k, v in changes.items():
            if k == "gravity":
                for c in range(3):
                    p.gravity[c] = float(v[c])
            else:
                setattr(p, k, v)
        _check(self._lib.mgsb_set_params(self.h, C.byref(p)), self.h)

    def set_fixed(self, mask, body: int = 0) -> None:
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        _check(self._lib.mgsb_set_fixed(self.h, body, _u8ptr(m)), self.h)

    def set_material(self, youngs, poisson, body: int = 0) -> None:
        T = self.num_tets(body)
        e = np.ascontiguousarray(np.broadcast_to(np.asarray(youngs, np.float32), (T,)))
        n = np.ascontiguousarray(np.broadcast_to(np.asarray(poisson, np.float32), (T,)))
        _check(self._lib.mgsb_set_material(self.h, body, _fptr(e), _fptr(n)), self.h)

    def set_capsule(self, a, b, radius: float, body: int = 0) -> None:
        aa = np.asarray(a, np.float32)
        bb = np.asarray(b, np.float32)
        _check(self._lib.mgsb_set_tool_capsule(self.h, body, _fptr(aa), _fptr(bb), float(radius)), self.h)

    def set_capsules(self, a, b, radius) -> None:
        aa = np.ascontiguousarray(a, np.float32)
        bb = np.ascontiguousarray(b, np.float32)
        rr = np.ascontiguousarray(radius, np.float32)
        _check(self._lib.mgsb_set_tool_capsules(self.h, _fptr(aa), _fptr(bb), _fptr(rr)), self.h)

    def set_spheres(self, centers, radii, active=None) -> None:
        c = np.ascontiguousarray(centers, np.float32).reshape(-1, 3)
        r = np.ascontiguousarray(radii, np.float32).reshape(-1)
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        _check(self._lib.mgsb_set_tool_spheres(self.h, c.shape[0], _fptr(c), _fptr(r),
                                               None if act is None else _u8ptr(act)), self.h)

    def set_state(self, positions=None, velocities=None, body: int = 0) -> None:
        p = None if positions is None else np.ascontiguousarray(positions, np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, np.float32)
        _check(self._lib.mgsb_set_state(self.h, body, None if p is None else _fptr(p),
                                        None if v is None else _fptr(v)), self.h)

    # -- stepping
    def step(self, n: int = 1) -> None:
        if n == 1:
            _check(self._lib.mgsb_step(self.h), self.h)
        else:
            _check(self._lib.mgsb_step_n(self.h, n), self.h)

    def synchronize(self) -> None:
        _check(self._lib.mgsb_synchronize(self.h), self.h)

    # -- outputs
    def positions(self, body: int = 0) -> np.ndarray:
        out = np.empty((self.num_verts(body), 3), np.float32)
        _check(self._lib.mgsb_get_positions(self.h, body, _fptr(out)), self.h)
        return out

    def all_positions(self) -> np.ndarray:
        n = sum(self.num_verts(b) for b in range(self.num_bodies))
        out = np.empty((n, 3), np.float32)
        _check(self._lib.mgsb_get_all_positions(self.h, _fptr(out)), self.h)
        return out

    def all_contact_flags(self) -> np.ndarray:
        n = sum(self.num_verts(b) for b in range(self.num_bodies))
        out = np.empty(n, np.int32)
        _check(self._lib.mgsb_get_all_contact_flags(self.h, _iptr(out)), self.h)
        return out

    def frame(self, positions: np.ndarray = None, contact_flags: np.ndarray = None):
        """Positions [sum V, 3] and contact flags [sum V] of every body in one readback (mgsb_get_frame);
        pass preallocated arrays to reuse them across frames."""
        n = getattr(self, "_nv_total", None)
        if n is None:
            n = self._nv_total = sum(self.num_verts(b) for b in range(self.num_bodies))
        if positions is None:
            positions = np.empty((n, 3), np.float32)
        if contact_flags is None:
            contact_flags = np.empty(n, np.int32)
        if positions.shape != (n, 3) or positions.dtype != np.float32 or not positions.flags.c_contiguous:
            raise ValueError("positions must be a C-contiguous float32 array of shape (%d, 3)" % n)
        if contact_flags.shape != (n,) or contact_flags.dtype != np.int32 or not contact_flags.flags.c_contiguous:
            raise ValueError("contact_flags must be a C-contiguous int32 array of shape (%d,)" % n)
        _check(self._lib.mgsb_get_frame(self.h, _fptr(positions), _iptr(contact_flags)), self.h)
        return positions, contact_flags

    def frame_view(self):
        """Positions [sum V, 3] and contact flags [sum V] as numpy views of the solver's pinned readback
        buffer (mgsb_get_frame_view): no host copy.  The views stay valid until the next readback call
        on this solver; copy them to keep a frame."""
        n = getattr(self, "_nv_total", None)
        if n is None:
            n = self._nv_total = sum(self.num_verts(b) for b in range(self.num_bodies))
        pp, fp = C.POINTER(C.c_float)(), C.POINTER(C.c_int32)()
        _check(self._lib.mgsb_get_frame_view(self.h, C.byref(pp), C.byref(fp)), self.h)
        if n == 0:
            return np.zeros((0, 3), np.float32), np.zeros(0, np.int32)
        return np.ctypeslib.as_array(pp, shape=(n, 3)), np.ctypeslib.as_array(fp, shape=(n,))

    def set_learned_smoother(self, net, guard_ratio: float = 0.5) -> None:
        """Attach a trained learned.MLP (None detaches); see mgsb_set_learned_smoother."""
        self._net = net   # keep the network alive while attached
        _check(self._lib.mgsb_set_learned_smoother(self.h, net.h if net is not None else None, guard_ratio), self.h)

    def learned_stats(self) -> tuple[int, int]:
        out = (C.c_uint64 * 2)()
        _check(self._lib.mgsb_learned_stats(self.h, out), self.h)
        return int(out[0]), int(out[1])

    def learned_cycle_norms(self) -> tuple[np.ndarray, np.ndarray]:
        """|r| before and after each learned V-cycle of the last frame (mgsb_learned_cycle_norms)."""
        n = C.c_int32()
        _check(self._lib.mgsb_learned_cycle_norms(self.h, None, None, 0, C.byref(n)), self.h)
        before, after = np.zeros(n.value), np.zeros(n.value)
        if n.value:
            dp = C.POINTER(C.c_double)
            _check(self._lib.mgsb_learned_cycle_norms(self.h, before.ctypes.data_as(dp), after.ctypes.data_as(dp),
                                                      n.value, C.byref(n)), self.h)
        return before, after

    def smoother_pairs(self, sweeps: int = 4) -> tuple[np.ndarray, np.ndarray]:
        """Training pairs (features [n,9], targets [n,3]) from the current state (mgsb_smoother_pairs)."""
        n = C.c_int64()
        cap = 3 * sum(self.num_verts(b) for b in range(self.num_bodies))
        x = np.empty((cap, 9), np.float32)
        t = np.empty((cap, 3), np.float32)
        _check(self._lib.mgsb_smoother_pairs(self.h, sweeps, _fptr(x), _fptr(t), cap, C.byref(n)), self.h)
        return x[: n.value], t[: n.value]

    def vcycle_residuals(self, cycles: int = 5, mode: int = 0) -> np.ndarray:
        """Residual norms of V-cycles on the last global step (mode 0 plain, 1 plain 1+1, 2 learned)."""
        out = np.empty(cycles + 1, np.float64)
        _check(self._lib.mgsb_vcycle_residuals(self.h, cycles, mode, out.ctypes.data_as(C.POINTER(C.c_double))), self.h)
        return out

    def positions_f64(self, body: int = 0) -> np.ndarray:
        out = np.empty((self.num_verts(body), 3), np.float64)
        _check(self._lib.mgsb_get_positions_f64(self.h, body, out.ctypes.data_as(C.POINTER(C.c_double))), self.h)
        return out

    def velocities(self, body: int = 0) -> np.ndarray:
        out = np.empty((self.num_verts(body), 3), np.float32)
        _check(self._lib.mgsb_get_velocities(self.h, body, _fptr(out)), self.h)
        return out

    def contact_flags(self, body: int = 0) -> np.ndarray:
        out = np.empty(self.num_verts(body), np.int32)
        _check(self._lib.mgsb_get_contact_flags(self.h, body, _iptr(out)), self.h)
        return out

    def contacts(self, body: int = 0) -> np.ndarray:
        n = C.c_size_t()
        _check(self._lib.mgsb_get_contacts(self.h, body, None, 0, C.byref(n)), self.h)
        out = np.empty(max(n.value, 1), np.int32)
        _check(self._lib.mgsb_get_contacts(self.h, body, _iptr(out), out.size, C.byref(n)), self.h)
        return out[: n.value]

    def collision_depth(self, body: int = 0) -> np.ndarray:
        out = np.empty(self.num_verts(body), np.float32)
        _check(self._lib.mgsb_get_collision_depth(self.h, body, _fptr(out)), self.h)
        return out

    def normals(self, body: int = 0) -> np.ndarray:
        out = np.empty((self.num_verts(body), 3), np.float32)
        _check(self._lib.mgsb_get_normals(self.h, body, _fptr(out)), self.h)
        return out

    def energy(self, body: int = 0) -> np.ndarray:
        out = np.empty(5, np.float64)
        _check(self._lib.mgsb_get_energy(self.h, body, out.ctypes.data_as(C.POINTER(C.c_double))), self.h)
        return out

    def device_positions_ptr(self, body: int = 0) -> int:
        p = C.POINTER(C.c_float)()
        _check(self._lib.mgsb_get_device_positions(self.h, body, C.byref(p)), self.h)
        return C.cast(p, C.c_void_p).value or 0

    def last_frame_ms(self) -> float:
        ms = C.c_float()
        _check(self._lib.mgsb_last_frame_ms(self.h, C.byref(ms)), self.h)
        return ms.value

    def launches_per_frame(self) -> int:
        n = C.c_int32()
        _check(self._lib.mgsb_launches_per_frame(self.h, C.byref(n)), self.h)
        return n.value

    def profile_frame(self) -> dict:
        """Run one frame with per-launch CUDA events: {kernel: (total_ms, launches)}."""
        cap = 64
        names = C.create_string_buffer(48 * cap)
        ms = np.zeros(cap, np.float32)
        cnt = np.zeros(cap, np.int32)
        n = C.c_int32()
        _check(self._lib.mgsb_profile_frame(self.h, cap, names, _fptr(ms), _iptr(cnt), C.byref(n)), self.h)
        raw = names.raw
        out = {}
        for k in range(min(n.value, cap)):
            nm = raw[48 * k: 48 * (k + 1)].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out

    def time_kernel(self, name: str, reps: int = 20) -> tuple:
        """Device time of one launch of kernel `name` inside the frame's
        launch chain (each of its launches repeated `reps` times back to
        back, no events in between): (us_per_launch, launches_per_frame).
        The state is restored afterwards; the simulation does not advance."""
        us = C.c_float()
        k = C.c_int32()
        _check(self._lib.mgsb_time_kernel(self.h, name.encode(), int(reps), C.byref(us), C.byref(k)), self.h)
        return float(us.value), int(k.value)

    def precompute(self) -> dict:
        T, V = self.num_tets(0), self.num_verts(0)
        inv = np.empty(9 * T, np.float32)
        ac = np.empty(12 * T, np.float32)
        vol = np.empty(T, np.float32)
        mass = np.empty(V, np.float32)
        diag = np.empty(V, np.float32)
        _check(self._lib.mgsb_get_precompute(self.h, _fptr(inv), _fptr(ac), _fptr(vol), _fptr(mass), _fptr(diag)),
               self.h)
        return dict(inv=inv.reshape(T, 9), ac=ac.reshape(T, 12), volume=vol, mass=mass, diag=diag)

    def level_info(self, level: int) -> dict:
        info = np.zeros(8, np.int32)
        _check(self._lib.mgsb_level_info(self.h, level, _iptr(info)), self.h)
        keys = ("n", "nnz", "nchild", "slice", "ell_entries", "cluster", "block", "fuse_l0")
        return {k: int(v) for k, v in zip(keys, info)}

    def body_level_size(self, body: int, level: int) -> int:
        """Rows of one body on one level (mgsb_body_level_size)."""
        n = C.c_int32()
        _check(self._lib.mgsb_body_level_size(self.h, body, level, C.byref(n)), self.h)
        return n.value

    def autotune(self, frames: int = 5) -> dict:
        """Pick the coarse-kernel shape by timing candidates; the state is restored."""
        ch = np.zeros(3, np.int32)
        _check(self._lib.mgsb_autotune(self.h, frames, _iptr(ch)), self.h)
        return {"cluster": int(ch[0]), "block": int(ch[1]), "fuse_l0": int(ch[2]), "split": self.coarse_split(),
                "dense_operator": self.coarse_dense()}

    def set_kernel_shape(self, cluster: int = 0, block: int = 0, fuse_level0: int = -1) -> None:
        _check(self._lib.mgsb_set_kernel_shape(self.h, cluster, block, fuse_level0), self.h)

    def set_coarse_split(self, split: int = 0) -> None:
        """Levels 1..split-1 grid-wide, the rest in the cluster kernel (0 = by size)."""
        _check(self._lib.mgsb_set_coarse_split(self.h, split), self.h)

    def set_surface_contact(self, triangles: bool = True) -> None:
        """Capsule against the surface triangles too (mgsb_set_surface_contact), or vertices only."""
        _check(self._lib.mgsb_set_surface_contact(self.h, 1 if triangles else 0), self.h)

    def set_coarse_dense(self, on: bool = True) -> None:
        """The dense coarse operator for the levels from the coarse split down (mgsb_set_coarse_dense)."""
        _check(self._lib.mgsb_set_coarse_dense(self.h, 1 if on else 0), self.h)

    def coarse_dense(self) -> bool:
        n = C.c_int32()
        _check(self._lib.mgsb_get_coarse_dense(self.h, C.byref(n)), self.h)
        return bool(n.value)

    def set_broad_phase(self, on: bool = True) -> None:
        """Uniform-grid broad phase for the capsule contact (same contacts as the all-vertex test)."""
        _check(self._lib.mgsb_set_broad_phase(self.h, 1 if on else 0), self.h)

    def set_fused_prolongation(self, on: bool = True) -> None:
        """Prolongation + first post-smoothing sweep as one kernel (default on)."""
        _check(self._lib.mgsb_set_fused_prolongation(self.h, 1 if on else 0), self.h)

    def set_fused_restriction(self, on: bool = True) -> None:
        """Level-1 restriction straight from level 0, no level-0 residual launch (default off)."""
        _check(self._lib.mgsb_set_fused_restriction(self.h, 1 if on else 0), self.h)

    def set_launch_overlap(self, on: bool = True) -> None:
        """Programmatic dependent launch between the frame's kernels (default on)."""
        _check(self._lib.mgsb_set_launch_overlap(self.h, 1 if on else 0), self.h)

    def coarse_split(self) -> int:
        v = np.zeros(1, np.int32)
        _check(self._lib.mgsb_get_coarse_split(self.h, _iptr(v)), self.h)
        return int(v[0])

    def level_size(self, level: int) -> tuple[int, int]:
        n = C.c_int32()
        z = C.c_int32()
        _check(self._lib.mgsb_level_size(self.h, level, C.byref(n), C.byref(z)), self.h)
        return n.value, z.value


class _LevelSolver(Solver):
    """A level of a TwoLevel handle: the Solver getters on a handle it does not own."""

    def __init__(self, lib, h, mesh, params):  # no Solver.__init__: the handle belongs to the TwoLevel
        self._lib = lib
        self.h = h
        self.meshes = [mesh]
        self.params = [params]

    def close(self) -> None:
        self.h = None


class TwoLevel:
    """The reference's two-level nested-iteration schedule (PDSolver_MG) on a coarse and a fine mesh of
    one body; levels[0] = fine, levels[1] = coarse (Solver getters)."""

    def __init__(self, coarse: TetMesh, fine: TetMesh, params: Params):
        self._lib = L.load()
        mc, kc = coarse.as_c()
        mf, kf = fine.as_c()
        h = C.c_void_p()
        st = self._lib.mgsb_mg2_create(C.byref(mc), C.byref(mf), C.byref(params), C.byref(h))
        if st != 0:
            msg = self._lib.mgsb_mg2_last_error(h) if h else b""
            raise MgsbError(st, "mgsb_mg2_create failed: " + (msg.decode() if msg else ""))
        self.h = h
        self.levels = []
        for lvl, mesh in ((0, fine), (1, coarse)):
            lh = C.c_void_p()
            _check(self._lib.mgsb_mg2_level(self.h, lvl, C.byref(lh)))
            self.levels.append(_LevelSolver(self._lib, lh, mesh, params))

    def _chk(self, st):
        if st != 0:
            msg = self._lib.mgsb_mg2_last_error(self.h)
            raise MgsbError(st, msg.decode() if msg else "")

    def set_fixed(self, coarse_mask=None, fine_mask=None) -> None:
        cm = np.ascontiguousarray(coarse_mask, np.uint8) if coarse_mask is not None else None
        fm = np.ascontiguousarray(fine_mask, np.uint8) if fine_mask is not None else None
        self._chk(self._lib.mgsb_mg2_set_fixed(self.h, _u8ptr(cm) if cm is not None else None,
                                               _u8ptr(fm) if fm is not None else None))

    def set_spheres(self, centers, radii, active=None) -> None:
        c = np.ascontiguousarray(centers, np.float32).reshape(-1, 3)
        r = np.ascontiguousarray(radii, np.float32).reshape(-1)
        a = np.ascontiguousarray(active, np.uint8) if active is not None else None
        self._chk(self._lib.mgsb_mg2_set_tool_spheres(self.h, c.shape[0], _fptr(c), _fptr(r),
                                                      _u8ptr(a) if a is not None else None))

    def step(self, n: int = 1) -> None:
        for _ in range(n):
            self._chk(self._lib.mgsb_mg2_step(self.h))

    def positions(self, level: int = 0) -> np.ndarray:
        return self.levels[level].positions()

    def close(self) -> None:
        if getattr(self, "h", None):
            for lv in self.levels:
                lv.close()
            self._lib.mgsb_mg2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
