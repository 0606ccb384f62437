"""Reference-faithful Jacobi/Chebyshev frame on the GPU (the drop-in for
PDSolver::Step) vs the FP64 oracle and vs the reference's own GPU frames."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle

from .golden.make_golden import TRAJ_ITERS, TRAJ_KEEP, traj_scene, traj_sphere_path

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _ref_pair(iters=TRAJ_ITERS, graph=1):
    m, fixed = traj_scene()
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI, iterations=iters, use_graph=graph)
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    return m, s, o


def test_ref_precompute_matches_oracle(lib, oracle_built):
    m, s, o = _ref_pair()
    a, b = s.precompute(), o.precompute()
    for k in ("inv", "ac", "volume", "mass", "diag"):
        err = np.abs(a[k].astype(np.float64) - b[k]).max() / np.abs(b[k]).max()
        assert err < 1e-6, (k, err)
    s.close()


def test_ref_frames_match_oracle(lib, oracle_built):
    """100 frames with a sphere pushed through the beam: max vertex error <= 5e-5 x bbox
    diagonal (the reference iteration amplifies FP32 rounding ~100x; see
    test_reference_iteration_sensitivity)."""
    m, s, o = _ref_pair()
    path = traj_sphere_path()
    tol = 5e-5 * m.bbox_diagonal()
    worst = 0.0
    flips = 0
    for f in range(path.shape[0]):
        for solver in (s, o):
            solver.set_spheres(path[f, :3][None], [path[f, 3]])
            solver.step()
        if f % 10 == 9:
            xg, xo = s.positions(), o.positions()
            worst = max(worst, np.abs(xg - xo).max())
            fg, fo = s.contact_flags(), o.contact_flags()
            diff = np.nonzero(fg != fo)[0]
            # a flag may only differ where the vertex sits on the threshold |x - c| = r
            d = np.linalg.norm(xo[diff] - path[f, :3][None].astype(np.float64), axis=1)
            assert np.all(np.abs(d - path[f, 3]) < 10 * tol), (f, diff)
            flips += len(diff)
    assert worst < tol, (worst, tol)
    s.close()


def test_ref_graph_equals_eager(lib):
    _, s1, _ = _ref_pair(iters=5, graph=1)
    _, s2, _ = _ref_pair(iters=5, graph=0)
    path = traj_sphere_path()
    for f in range(30):
        for s in (s1, s2):
            s.set_spheres(path[f, :3][None], [path[f, 3]])
            s.step()
    assert np.array_equal(s1.positions(), s2.positions())


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "ref_traj.npz")), reason="GPU golden not generated")
def test_ref_frames_match_reference_gpu(lib):
    """Against PDSolver::Step of the reference itself (fixture made on a B200)."""
    g = np.load(os.path.join(GOLDEN, "ref_traj.npz"))
    m, s, _ = _ref_pair()
    path = traj_sphere_path()
    tol = 5e-5 * m.bbox_diagonal()
    for f in range(path.shape[0]):
        s.set_spheres(path[f, :3][None], [path[f, 3]])
        s.step()
        if f in TRAJ_KEEP:
            k = TRAJ_KEEP.index(f)
            err = np.abs(s.positions() - g["positions"][k]).max()
            assert err < tol, (f, err)
    s.close()


def test_pdsolver_mirror(lib):
    """The reference-shaped interface: fields, Init, SetFixedVert by fixer spheres, Step."""
    m, _ = traj_scene()
    mg.extract_surface(m)
    solver = mg.PDSolver()
    solver.m_iterNum = 10
    solver.m_sphereFixers = [mg.SphereFixer((0.0, 7.0, 0.0), 1.5)]
    solver.m_sphereColliders = [mg.SphereCollider((2.5, -3.0, 0.2), 0.8)]
    solver.Init(m.positions.reshape(-1), m.tets.reshape(-1), m.tris.reshape(-1), m.tri_opposite)
    assert (solver.m_tetVertFixed == 0).sum() > 0
    for _ in range(40):
        solver.m_sphereColliders[0].MoveDelta((-0.05, 0.0, 0.0))
        solver.Step()
    x = solver.m_tetVertPos.reshape(-1, 3)
    assert np.isfinite(x).all()
    fixed = solver.m_tetVertFixed == 0
    assert np.abs(x[fixed] - m.positions[fixed]).max() == 0.0
    assert solver.m_tetVertIsCollide.sum() > 0
