"""mgsb_get_normals_noalloc (the allocation-free normals readback) called
through the C ABI, against mgsb_get_normals on the same solver state."""
import ctypes as C

import numpy as np
import pytest

import multigridsoftbody_b200 as mg

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu

MGSB_OK, MGSB_INVALID_ARG, MGSB_NOT_SUPPORTED = 0, 1, 6


def _call(lib, name, solver, num_verts, body=0):
    out = np.full((num_verts, 3), np.nan, np.float32)
    status = getattr(lib, name)(solver.h, body, out.ctypes.data_as(C.POINTER(C.c_float)))
    return status, out


def test_noalloc_normals_equal_allocating_path(lib):
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    path = capsule_path(24, start=(0.0, 0.0, 1.3))
    for f in range(24):
        s.set_capsule(*path[f], 0.3)
        s.step()
        if f not in (11, 23):
            continue
        st_ref, ref = _call(lib, "mgsb_get_normals", s, m.num_verts)
        assert st_ref == MGSB_OK
        for _ in range(2):                      # two calls in a row
            st, got = _call(lib, "mgsb_get_normals_noalloc", s, m.num_verts)
            assert st == MGSB_OK, lib.mgsb_last_error_string(s.h)
            assert np.abs(got - ref).max() <= 1e-6
    s.close()


def test_noalloc_normals_batch_and_limits(lib):
    m0, f0 = beam(4, 40, 4)
    m1, f1 = beam(3, 20, 5, half_len=5.0)
    s = mg.Solver([m0, m1], mg_params(levels=3))
    s.set_fixed(f0, body=0)
    s.set_fixed(f1, body=1)
    # a pending set-up is not rebuilt by the allocation-free call
    st, _ = _call(lib, "mgsb_get_normals_noalloc", s, m1.num_verts, body=1)
    assert st == MGSB_INVALID_ARG
    s.step(4)
    for body, m in ((0, m0), (1, m1)):
        _, ref = _call(lib, "mgsb_get_normals", s, m.num_verts, body)
        st, got = _call(lib, "mgsb_get_normals_noalloc", s, m.num_verts, body)
        assert st == MGSB_OK and np.abs(got - ref).max() <= 1e-6
    s.close()
    # 128 x 128 x 1 plate: 66,560 surface triangles, above the 65,536 the scratch holds
    plate = mg.box_mesh(128, 128, 1, (-8.0, -8.0, -0.0625), (8.0, 8.0, 0.0625))
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    s = mg.Solver(plate, p)
    s.step()
    st, _ = _call(lib, "mgsb_get_normals_noalloc", s, plate.num_verts)
    assert st == MGSB_NOT_SUPPORTED
    assert b"65536" in lib.mgsb_last_error_string(s.h)
    st, ref = _call(lib, "mgsb_get_normals", s, plate.num_verts)
    assert st == MGSB_OK and np.isfinite(ref).all()
    s.close()
