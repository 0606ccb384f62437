"""ctypes binding of the FP64 oracle (oracle/mgsb_oracle.h) — test infrastructure only."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libmgsb_oracle.so")


def build_oracle() -> str:
    res = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    return ORACLE_LIB


_lib = None
_FP = C.POINTER(C.c_float)
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_LIB):
        build_oracle()
    lib = C.CDLL(ORACLE_LIB)
    sig = {
        "oracle_create": (C.c_void_p, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]),
        "oracle_destroy": (None, [C.c_void_p]),
        "oracle_set_fixed": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
        "oracle_set_material": (C.c_int, [C.c_void_p, _FP, _FP]),
        "oracle_set_tool_capsule": (C.c_int, [C.c_void_p, _FP, _FP, C.c_float]),
        "oracle_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
        "oracle_set_surface_contact": (C.c_int, [C.c_void_p, C.c_int]),
        "oracle_segment_triangle": (C.c_double, [_DP, _DP, _DP, _DP]),
        "oracle_set_tool_spheres": (C.c_int, [C.c_void_p, C.c_int32, _FP, _FP, C.POINTER(C.c_uint8)]),
        "oracle_step": (C.c_int, [C.c_void_p]),
        "oracle_num_verts": (C.c_int, [C.c_void_p]),
        "oracle_get_positions": (None, [C.c_void_p, _DP]),
        "oracle_get_velocities": (None, [C.c_void_p, _DP]),
        "oracle_get_contact_flags": (None, [C.c_void_p, _IP]),
        "oracle_get_collision_depth": (None, [C.c_void_p, _DP]),
        "oracle_set_state": (None, [C.c_void_p, _DP, _DP]),
        "oracle_get_precompute": (None, [C.c_void_p, _DP, _DP, _DP, _DP, _DP]),
        "oracle_get_energy": (None, [C.c_void_p, _DP]),
        "oracle_last_residual": (C.c_double, [C.c_void_p]),
        "oracle_set_threads": (C.c_int, [C.c_int]),
        "oracle_level_size": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP]),
        "oracle_level_prolongation": (C.c_int, [C.c_void_p, C.c_int, _IP, _DP]),
        "oracle_level_matrix": (C.c_int, [C.c_void_p, C.c_int, _DP, _IP, _IP, _DP]),
        "oracle_surface_normals": (None, [_DP, C.c_int32, _IP, C.c_int32, _DP]),
        "oracle_mlp_forward": (None, [_DP, _DP, C.c_int32, C.c_int32, _DP]),
        "oracle_mg2_create": (C.c_void_p, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]),
        "oracle_mg2_destroy": (None, [C.c_void_p]),
        "oracle_mg2_level": (C.c_void_p, [C.c_void_p, C.c_int]),
        "oracle_mg2_step": (None, [C.c_void_p]),
        "oracle_mlp_loss_grad": (C.c_double, [_DP, _DP, _DP, C.c_int32, C.c_int32, _DP]),
        "oracle_ref_rotation": (None, [_DP, _DP]),
        "oracle_svd_rotation": (None, [_DP, _DP]),
        "oracle_inverse3": (C.c_double, [_DP, _DP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def set_threads(n: int = 0) -> int:
    """Host threads of the oracle's OpenMP loops (0: all); returns the count in force."""
    return int(_load().oracle_set_threads(int(n)))


def _dp(a):
    return a.ctypes.data_as(_DP)


class Oracle:
    """FP64 restatement of the frame; mirrors the product's Solver interface."""

    def __init__(self, mesh, params):
        from multigridsoftbody_b200.api import TetMesh  # mesh container only
        assert isinstance(mesh, TetMesh)
        self._lib = _load()
        self.mesh = mesh
        m, self._keep = mesh.as_c()
        err = C.create_string_buffer(256)
        self._params = params
        self.h = self._lib.oracle_create(C.byref(m), C.byref(params), err, 256)
        if not self.h:
            raise RuntimeError("oracle_create: " + err.value.decode())
        self.V = mesh.num_verts
        self.T = mesh.num_tets

    def close(self):
        if getattr(self, "h", None):
            self._lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fixed(self, mask):
        m = np.ascontiguousarray(mask, np.uint8)
        self._lib.oracle_set_fixed(self.h, m.ctypes.data_as(C.POINTER(C.c_uint8)))

    def set_material(self, youngs, poisson):
        e = np.ascontiguousarray(np.broadcast_to(np.asarray(youngs, np.float32), (self.T,)))
        n = np.ascontiguousarray(np.broadcast_to(np.asarray(poisson, np.float32), (self.T,)))
        self._lib.oracle_set_material(self.h, e.ctypes.data_as(_FP), n.ctypes.data_as(_FP))

    def set_params(self, params):
        self._params = params
        st = self._lib.oracle_set_params(self.h, C.byref(params))
        if st != 0:
            raise RuntimeError(f"oracle_set_params: status {st}")

    def set_surface_contact(self, triangles=True):
        self._lib.oracle_set_surface_contact(self.h, 1 if triangles else 0)

    def set_capsule(self, a, b, radius):
        aa = np.asarray(a, np.float32)
        bb = np.asarray(b, np.float32)
        self._lib.oracle_set_tool_capsule(self.h, aa.ctypes.data_as(_FP), bb.ctypes.data_as(_FP), float(radius))

    def set_spheres(self, centers, radii, active=None):
        c = np.ascontiguousarray(centers, np.float32).reshape(-1, 3)
        r = np.ascontiguousarray(radii, np.float32).reshape(-1)
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        self._lib.oracle_set_tool_spheres(self.h, c.shape[0], c.ctypes.data_as(_FP), r.ctypes.data_as(_FP),
                                          None if act is None else act.ctypes.data_as(C.POINTER(C.c_uint8)))

    def step(self, n=1):
        for _ in range(n):
            st = self._lib.oracle_step(self.h)
            if st != 0:
                raise RuntimeError(f"oracle_step status {st}")

    def positions(self):
        out = np.empty((self.V, 3), np.float64)
        self._lib.oracle_get_positions(self.h, _dp(out))
        return out

    def velocities(self):
        out = np.empty((self.V, 3), np.float64)
        self._lib.oracle_get_velocities(self.h, _dp(out))
        return out

    def contact_flags(self):
        out = np.empty(self.V, np.int32)
        self._lib.oracle_get_contact_flags(self.h, out.ctypes.data_as(_IP))
        return out

    def collision_depth(self):
        out = np.empty(self.V, np.float64)
        self._lib.oracle_get_collision_depth(self.h, _dp(out))
        return out

    def set_state(self, positions=None, velocities=None):
        p = None if positions is None else np.ascontiguousarray(positions, np.float64)
        v = None if velocities is None else np.ascontiguousarray(velocities, np.float64)
        self._lib.oracle_set_state(self.h, None if p is None else _dp(p), None if v is None else _dp(v))

    def precompute(self):
        inv = np.empty(9 * self.T)
        ac = np.empty(12 * self.T)
        vol = np.empty(self.T)
        mass = np.empty(self.V)
        diag = np.empty(self.V)
        self._lib.oracle_get_precompute(self.h, _dp(inv), _dp(ac), _dp(vol), _dp(mass), _dp(diag))
        return dict(inv=inv.reshape(-1, 9), ac=ac.reshape(-1, 12), volume=vol, mass=mass, diag=diag)

    def energy(self):
        out = np.empty(5)
        self._lib.oracle_get_energy(self.h, _dp(out))
        return out

    def last_residual(self):
        return float(self._lib.oracle_last_residual(self.h))

    def level_size(self, level):
        n = C.c_int32()
        z = C.c_int32()
        st = self._lib.oracle_level_size(self.h, level, C.byref(n), C.byref(z))
        if st != 0:
            raise RuntimeError("bad level")
        return n.value, z.value

    def level_prolongation(self, level, n_finer):
        ids = np.empty(4 * n_finer, np.int32)
        w = np.empty(4 * n_finer)
        self._lib.oracle_level_prolongation(self.h, level, ids.ctypes.data_as(_IP), _dp(w))
        return ids.reshape(-1, 4), w.reshape(-1, 4)

    def level_matrix(self, level):
        n, z = self.level_size(level)
        diag = np.empty(n)
        ptr = np.empty(n + 1, np.int32)
        col = np.empty(max(z, 1), np.int32)
        val = np.empty(max(z, 1))
        self._lib.oracle_level_matrix(self.h, level, _dp(diag), ptr.ctypes.data_as(_IP), col.ctypes.data_as(_IP),
                                      _dp(val))
        return diag, ptr, col[:z], val[:z]


def ref_rotation(F):
    lib = _load()
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    R = np.empty(9)
    lib.oracle_ref_rotation(_dp(F), _dp(R))
    return R.reshape(3, 3)


def svd_rotation(F):
    lib = _load()
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    R = np.empty(9)
    lib.oracle_svd_rotation(_dp(F), _dp(R))
    return R.reshape(3, 3)


def segment_triangle(p0, p1, a, b, c):
    """Distance between segment p0p1 and triangle abc, and the closest points (on the segment, on the
    triangle)."""
    seg = np.ascontiguousarray(np.concatenate([p0, p1]), np.float64)
    tri = np.ascontiguousarray(np.concatenate([a, b, c]), np.float64)
    q = np.zeros(3)
    h = np.zeros(3)
    d = _load().oracle_segment_triangle(_dp(seg), _dp(tri), _dp(q), _dp(h))
    return d, q, h


def surface_normals(positions, tris):
    """Vertex normals of the triangle surface `tris` [F,3] at `positions` [V,3]."""
    lib = _load()
    pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    out = np.empty_like(pos)
    lib.oracle_surface_normals(_dp(pos), pos.shape[0], t.ctypes.data_as(_IP), t.shape[0], _dp(out))
    return out


def mlp_forward(params, x, bf16=True):
    """Learned-smoother MLP on rows of x [n, 9] -> [n, 3] (FP64, optional BF16 rounding)."""
    lib = _load()
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 9)
    y = np.empty((x.shape[0], 3))
    lib.oracle_mlp_forward(_dp(p), _dp(x), x.shape[0], int(bf16), _dp(y))
    return y


def mlp_loss_grad(params, x, t, bf16=True):
    lib = _load()
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 9)
    t = np.ascontiguousarray(t, np.float64).reshape(-1, 3)
    g = np.empty(p.shape[0])
    loss = lib.oracle_mlp_loss_grad(_dp(p), _dp(x), _dp(t), x.shape[0], int(bf16), _dp(g))
    return float(loss), g


class _Level(Oracle):
    """One level of an OracleTwoLevel (borrowed handle)."""

    def __init__(self, lib, h, mesh):  # noqa: D401 - no Oracle.__init__: the handle is owned by the pair
        self._lib = lib
        self.h = h
        self.mesh = mesh
        self.V = mesh.num_verts
        self.T = mesh.num_tets

    def close(self):
        self.h = None


class OracleTwoLevel:
    """FP64 restatement of the reference's two-level schedule (PDSolver_MG); level 0 = fine, 1 = coarse."""

    def __init__(self, coarse, fine, params):
        self._lib = _load()
        mc, self._kc = coarse.as_c()
        mf, self._kf = fine.as_c()
        err = C.create_string_buffer(256)
        self._params = params
        self.h = self._lib.oracle_mg2_create(C.byref(mc), C.byref(mf), C.byref(params), err, 256)
        if not self.h:
            raise RuntimeError("oracle_mg2_create: " + err.value.decode())
        self.levels = [_Level(self._lib, self._lib.oracle_mg2_level(self.h, 0), fine),
                       _Level(self._lib, self._lib.oracle_mg2_level(self.h, 1), coarse)]

    def set_fixed(self, coarse_mask, fine_mask):
        self.levels[1].set_fixed(coarse_mask)
        self.levels[0].set_fixed(fine_mask)

    def set_spheres(self, centers, radii, active=None):
        for lv in self.levels:
            lv.set_spheres(centers, radii, active)

    def step(self, n=1):
        for _ in range(n):
            self._lib.oracle_mg2_step(self.h)

    def positions(self, level=0):
        return self.levels[level].positions()

    def contact_flags(self, level=0):
        return self.levels[level].contact_flags()

    def close(self):
        if getattr(self, "h", None):
            self._lib.oracle_mg2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
