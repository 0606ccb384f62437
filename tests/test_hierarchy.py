"""The product's multigrid hierarchy (host-built, inspected without a GPU through
mgsb_inspect_level) against the oracle's independent construction."""
import ctypes as C

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200 import _lib as L
from oracle.binding import Oracle

from .common import beam, mg_params


def inspect(lib, mesh, params, fixed, level):
    cm, keep = mesh.as_c()
    fx = np.ascontiguousarray(fixed, np.uint8)
    n, z = C.c_int32(), C.c_int32()
    st = lib.mgsb_inspect_level(C.byref(cm), C.byref(params), fx.ctypes.data_as(C.POINTER(C.c_uint8)), level,
                                C.byref(n), C.byref(z), None, None, None, None, None, None)
    assert st == 0
    nf = mesh.num_verts if level == 1 else None
    out = {"n": n.value, "nnz": z.value}
    diag = np.empty(n.value, np.float32)
    ptr = np.empty(n.value + 1, np.int32)
    col = np.empty(max(z.value, 1), np.int32)
    val = np.empty(max(z.value, 1), np.float32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    if level > 0:
        # rows of the prolongation = vertices of the next finer level
        prev = inspect(lib, mesh, params, fixed, level - 1)["n"] if level > 1 else mesh.num_verts
        pid = np.empty(4 * prev, np.int32)
        pw = np.empty(4 * prev, np.float32)
    else:
        pid = pw = None
    st = lib.mgsb_inspect_level(C.byref(cm), C.byref(params), fx.ctypes.data_as(C.POINTER(C.c_uint8)), level,
                                C.byref(n), C.byref(z), None if pid is None else ip(pid),
                                None if pw is None else fp(pw), fp(diag), ip(ptr), ip(col), fp(val))
    assert st == 0
    out.update(diag=diag, ptr=ptr, col=col[: z.value], val=val[: z.value])
    if pid is not None:
        out.update(pid=pid.reshape(-1, 4), pw=pw.reshape(-1, 4))
    return out


@pytest.mark.parametrize("dims,levels", [((4, 40, 4), 3), ((3, 30, 3), 3), ((12, 120, 12), 4)])
def test_hierarchy_matches_oracle(lib, oracle_built, dims, levels):
    m, fixed = beam(*dims)
    p = mg_params(levels=levels)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    for l in range(levels):
        h = inspect(lib, m, p, fixed, l)
        diag, ptr, col, val = o.level_matrix(l)
        assert h["n"] == len(diag) and h["nnz"] == len(col), l
        scale = np.abs(diag).max()
        assert np.abs(h["diag"] - diag).max() <= 1e-6 * scale, l
        assert np.array_equal(h["ptr"], ptr), l
        assert np.array_equal(h["col"], col), l
        assert np.abs(h["val"] - val).max() <= 1e-6 * scale, l
        if l > 0:
            n_prev = len(h["pid"])
            ids, w = o.level_prolongation(l, n_prev)
            assert np.abs(h["pw"] - w).max() < 1e-6, l
            nz = w > 0
            assert np.array_equal(h["pid"][nz], ids[nz]), l


def test_inspect_rejects_bad_level(lib):
    m, fixed = beam(2, 10, 2)
    p = mg_params(levels=2)
    cm, keep = m.as_c()
    n, z = C.c_int32(), C.c_int32()
    assert lib.mgsb_inspect_level(C.byref(cm), C.byref(p), None, 5, C.byref(n), C.byref(z), None, None, None, None,
                                  None, None) == 1
