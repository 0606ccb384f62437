"""Diagnostics on the device vs the oracle: surface vertex normals
(UpdateTriNormal + AvgOutsideTetVertNormal) and the energy/convergence
reduction (runCalEnergy) for the three solver kinds."""
import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle, surface_normals

from .common import beam, capsule_path, mg_params
from .golden.make_golden import TRAJ_ITERS, traj_scene, traj_sphere_path

pytestmark = pytest.mark.gpu


def _normals_check(s, m, body=0):
    mg.extract_surface(m)
    x = s.positions(body).astype(np.float64)
    got = s.normals(body)
    want = surface_normals(x, m.tris)
    on_surface = np.zeros(m.num_verts, bool)
    on_surface[m.tris.reshape(-1)] = True
    assert np.all(got[~on_surface] == 0.0)
    assert np.abs(got - want).max() < 1e-5, np.abs(got - want).max()
    assert np.allclose(np.linalg.norm(got[on_surface], axis=1), 1.0, atol=1e-5)


def test_normals_match_oracle_after_contact(lib, oracle_built):
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    _normals_check(s, m)                         # rest state
    for a, b in capsule_path(30, start=(0.0, 0.0, 1.3)):
        s.set_capsule(a, b, 0.3)
        s.step()
    _normals_check(s, m)                         # deformed by gravity and the capsule


def test_normals_batch_body(lib, oracle_built):
    m0, f0 = beam(4, 40, 4)
    m1, f1 = beam(3, 20, 5, half_len=5.0)
    s = mg.Solver([m0, m1], mg_params(levels=3))
    s.set_fixed(f0, body=0)
    s.set_fixed(f1, body=1)
    s.step(8)
    _normals_check(s, m0, body=0)
    _normals_check(s, m1, body=1)


def _energy_pair(kind_params, m, fixed, frames, tool):
    s = mg.Solver(m, kind_params)
    s.set_fixed(fixed)
    o = Oracle(m, kind_params)
    o.set_fixed(fixed)
    for f in range(frames):
        for solver in (s, o):
            tool(solver, f)
            solver.step()
    return s.energy(), o.energy()


def _assert_energy(got, want, rtol):
    # Ek, Ep, Ec relative; contact count exact
    for k in range(3):
        assert abs(got[k] - want[k]) <= rtol * max(abs(want[k]), 1e-12), (k, got, want)
    assert got[3] == want[3], (got, want)


def _capsule_energy(precision, passes):
    m, fixed = beam(4, 40, 4)
    path = capsule_path(40, start=(0.0, 0.0, 1.3))
    p = mg_params(levels=3, precision=precision, refinement_passes=passes)
    return _energy_pair(p, m, fixed, 40, lambda sv, f: sv.set_capsule(*path[f], 0.3))


def test_energy_multigrid(lib, oracle_built):
    """Ek, Ep, Ec and the contact count follow the state, so they match the
    oracle to the trajectory's accuracy.  The residual norm of the last global
    step measures each solver's own convergence: in FP32 it sits at the
    rounding floor of the contact terms (c = 1e6), mixed precision (FP64
    residual, 2 refinement passes) brings it well below that, and the FP64
    oracle lower still."""
    got32, want32 = _capsule_energy(mg.PRECISION_FP32, 1)
    got_mx, want_mx = _capsule_energy(mg.PRECISION_MIXED, 2)
    for got, want in ((got32, want32), (got_mx, want_mx)):
        assert want[3] > 0 and want[2] > 0
        _assert_energy(got, want, rtol=1e-4)
    assert 0 < got32[4] < 1e-2 and want32[4] < got32[4]
    assert 0 < got_mx[4] < got32[4] / 10 and want_mx[4] < got_mx[4]


def test_energy_reference_kind(lib, oracle_built):
    """The reference kind's last term is |x - prev| of the last iteration."""
    m, fixed = traj_scene()
    path = traj_sphere_path()
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI, iterations=TRAJ_ITERS)
    got, want = _energy_pair(p, m, fixed, 30, lambda sv, f: sv.set_spheres(path[f, :3][None], [path[f, 3]]))
    assert want[3] > 0 and want[2] > 0
    _assert_energy(got, want, rtol=2e-2)
    assert abs(got[4] - want[4]) <= 2e-2 * want[4], (got, want)


def test_energy_before_first_frame(lib):
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    e = s.energy()
    assert np.all(np.abs(e) < 1e-8), e           # at rest: no motion, strain, contact or residual
