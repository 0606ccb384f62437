"""mgsb_set_params through the C ABI: parameters changed between frames (the
reference's public fields m_iterNum, m_dt, m_damping, m_volumnStiffness,
m_collisionStiffness, m_rho, m_gravity{X,Y,Z}, PDSolver.h:72-81, assigned after
Init) take effect on the next frame, exactly as if the solver had been created
with them, and invalid or fixed-at-create changes are refused unchanged."""
import ctypes as C

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200 import _lib as L
from oracle.binding import Oracle

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu


def _changed(p):
    q = L.Params.from_buffer_copy(p)
    q.iterations = 6
    q.dt = 1.0 / 120.0
    q.damping = 0.9
    q.gravity[0], q.gravity[1], q.gravity[2] = 0.0, 0.0, -5.0
    return q


def test_set_params_multigrid_matches_fresh_solver_and_oracle(lib, oracle_built):
    """FP32 multigrid: 6 frames, then new dt, iterations, damping, gravity, sweeps and Young's modulus via
    mgsb_set_params, 6 more frames.  Equals a solver created with the new parameters from the same state,
    and the FP64 oracle given the same change, within 1e-5 x bbox diagonal with the same contacts."""
    m, fixed = beam(4, 40, 4)
    p0 = mg_params(levels=3)
    p1 = _changed(p0)
    p1.pre_sweeps, p1.post_sweeps = 1, 1
    p1.youngs_modulus = 2e5
    path = capsule_path(12, start=(0.0, 0.0, 1.3))
    a = mg.Solver(m, p0)
    a.set_fixed(fixed)
    o = Oracle(m, p0)
    o.set_fixed(fixed)
    for f in range(6):
        for x in (a, o):
            x.set_capsule(*path[f], 0.3)
            x.step()
    x6, v6 = a.positions(), a.velocities()
    a.set_params(p1)
    o.set_params(p1)
    got = a.get_params()
    assert got.iterations == 6 and got.pre_sweeps == 1 and abs(got.dt - 1 / 120) < 1e-9 and got.gravity[2] == -5.0
    b = mg.Solver(m, p1)
    b.set_fixed(fixed)
    b.set_state(x6, v6)
    for f in range(6, 12):
        for x in (a, b, o):
            x.set_capsule(*path[f], 0.3)
            x.step()
    tol = 1e-5 * m.bbox_diagonal()
    assert np.array_equal(a.positions(), b.positions())
    assert np.abs(a.positions() - o.positions()).max() < tol
    assert np.array_equal(a.contact_flags(), o.contact_flags())
    assert a.contact_flags().sum() > 0
    # the new material really applies: the stiffer beam sags less than one that kept E = 1e5
    c = mg.Solver(m, p0)
    c.set_fixed(fixed)
    c.set_state(x6, v6)
    c.set_params(_changed(p0))
    for f in range(6, 12):
        c.set_capsule(*path[f], 0.3)
        c.step()
    assert not np.array_equal(c.positions(), a.positions())
    for x in (a, b, c):
        x.close()


def test_set_params_refused_unchanged(lib):
    m, fixed = beam(4, 40, 4)
    p0 = mg_params(levels=3)
    s = mg.Solver(m, p0)
    s.set_fixed(fixed)
    s.step()
    for field, value, status in (("dt", -1.0, "invalid argument"), ("levels", 1, "invalid argument"),
                                 ("precision", mg.PRECISION_MIXED, "not supported"),
                                 ("solver", mg.SOLVER_REFERENCE_JACOBI, "not supported")):
        q = L.Params.from_buffer_copy(p0)
        setattr(q, field, value)
        with pytest.raises(mg.MgsbError) as ei:
            s.set_params(q)
        assert status in str(ei.value), (field, str(ei.value))
        assert getattr(s.get_params(), field) == getattr(p0, field)
    s.step()
    assert np.isfinite(s.positions()).all()
    s.close()


def test_pdsolver_fields_after_init(lib):
    """The reference mirror: m_iterNum / m_dt / m_damping / m_gravity* assigned after Init act on the next
    Step, like a PDSolver initialised with those values from the same state."""
    m, fixed = beam(4, 40, 4)
    a = mg.PDSolver()
    a.Init(m.positions, m.tets)
    a._solver.set_fixed(fixed)
    for _ in range(3):
        a.Step()
    x3, v3 = a.solver.positions(), a.solver.velocities()
    a.m_iterNum, a.m_dt, a.m_damping, a.m_gravityZ = 12, 1.0 / 90.0, 0.97, -2.0
    b = mg.PDSolver()
    b.m_iterNum, b.m_dt, b.m_damping, b.m_gravityZ = 12, 1.0 / 90.0, 0.97, -2.0
    b.Init(m.positions, m.tets)
    b._solver.set_fixed(fixed)
    b.solver.set_state(x3, v3)
    for _ in range(4):
        a.Step()
        b.Step()
    assert a.solver.get_params().iterations == 12
    assert np.array_equal(a.m_tetVertPos, b.m_tetVertPos)
