"""The FP64 oracle pinned against the reference's own outputs (golden fixtures
generated by tests/golden/make_golden.py from the reference compiled headless),
plus structural properties of its multigrid hierarchy.  CPU only."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle, ref_rotation, svd_rotation

from .common import beam, mg_params

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_precompute_matches_reference(oracle_built, golden_cpu):
    """PDSolver::InitVolumeConstraint (FP32 in the reference) vs the FP64 restatement."""
    g = golden_cpu
    m = mg.TetMesh(g["pre_pos"], g["pre_tets"])
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    o = Oracle(m, p)
    pre = o.precompute()
    for key, gk in [("inv", "pre_inv"), ("ac", "pre_ac"), ("volume", "pre_vol"), ("mass", "pre_mass"),
                    ("diag", "pre_diag")]:
        ref = g[gk].astype(np.float64)
        err = np.abs(pre[key] - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err < 2e-5, (key, err)


def test_ref_rotation_matches_reference(oracle_built, golden_cpu):
    F, R = golden_cpu["rot_F"], golden_cpu["rot_R"]
    for k in range(len(F)):
        Ro = ref_rotation(F[k])
        assert np.abs(Ro - R[k]).max() < 2e-5, k


def test_svd_rotation_matches_reference(oracle_built, golden_cpu):
    """The rotation-variant SVD equals the reference's polar rotation for det F > 0."""
    F, R = golden_cpu["rot_F"], golden_cpu["rot_R"]
    for k in range(len(F)):
        Rs = svd_rotation(F[k])
        assert np.abs(Rs - R[k]).max() < 2e-5, k
        assert abs(np.linalg.det(Rs) - 1) < 1e-12
        assert np.abs(Rs.T @ Rs - np.eye(3)).max() < 1e-12


def test_svd_rotation_inverted(oracle_built):
    F = np.diag([1.2, 0.9, -0.3])
    R = svd_rotation(F)
    assert np.abs(R - np.eye(3)).max() < 1e-12   # closest rotation flips the smallest axis
    assert abs(np.linalg.det(svd_rotation(np.diag([2.0, -1.0, 0.5]))) - 1) < 1e-12


def test_inverse_matches_reference(oracle_built, golden_cpu):
    from oracle.binding import _load, _dp
    lib = _load()
    for A, Ri, d in zip(golden_cpu["inv_A"], golden_cpu["inv_R"], golden_cpu["inv_det"]):
        R = np.empty(9)
        det = lib.oracle_inverse3(_dp(np.ascontiguousarray(A.reshape(9), np.float64)), _dp(R))
        assert abs(det - d) < 1e-5 * max(1, abs(d))
        assert np.abs(R.reshape(3, 3) - Ri).max() < 1e-4 * max(1, np.abs(Ri).max())


def test_hierarchy_properties(oracle_built):
    m, fixed = beam(4, 40, 4)
    o = Oracle(m, mg_params(levels=3))
    o.set_fixed(fixed)
    sizes = [o.level_size(l)[0] for l in range(3)]
    assert sizes == [1025, 189, 44]
    n_prev = 1025
    for l in (1, 2):
        ids, w = o.level_prolongation(l, n_prev)
        rows = w.sum(1)
        active_rows = rows > 0
        assert np.allclose(rows[active_rows], 1.0, atol=1e-12)
        assert (w >= 0).all()
        if l == 1:
            assert not active_rows[fixed.astype(bool)].any()   # fixed rows are zero
        diag, ptr, col, val = o.level_matrix(l)
        n = len(diag)
        A = np.zeros((n, n))
        A[np.arange(n), np.arange(n)] = diag
        for i in range(n):
            A[i, col[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
        assert np.abs(A - A.T).max() <= 1e-9 * np.abs(A).max()
        ev = np.linalg.eigvalsh(A[diag > 0][:, diag > 0])
        assert ev.min() > 0
        n_prev = n


def test_mg_residual_and_energy(oracle_built):
    """Plain MG: the residual after a frame is tiny and Ep stays finite under gravity."""
    m, fixed = beam(4, 40, 4)
    o = Oracle(m, mg_params(levels=3))
    o.set_fixed(fixed)
    for _ in range(10):
        o.step()
    assert o.last_residual() < 1e-3
    e = o.energy()
    assert np.isfinite(e).all() and e[1] > 0
    x = o.positions()
    assert np.abs(x[fixed.astype(bool)] - m.positions[fixed.astype(bool)]).max() == 0.0


def test_planted_mistake_is_detected(oracle_built):
    """A parity comparison must fail when the oracle is run with a wrong constant."""
    m, fixed = beam(2, 10, 2)
    good = Oracle(m, mg_params(levels=2))
    bad = Oracle(m, mg_params(levels=2, youngs_modulus=1.01e5))   # 1 % stiffer material
    for o in (good, bad):
        o.set_fixed(fixed)
        o.step(30)
    diag = m.bbox_diagonal()
    assert np.abs(good.positions() - bad.positions()).max() > 1e-5 * diag


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "ref_traj.npz")), reason="GPU golden not generated")
def test_oracle_ref_mode_matches_reference_trajectory(oracle_built):
    """FP64 restatement of PDSolver::Step vs the reference's own GPU frames.

    Tolerance 5e-5 x bbox diagonal: the reference's 20-iteration Jacobi/Chebyshev
    frame amplifies a 1e-6 perturbation of the state to ~1e-4 within a few frames
    (measured), so FP32 rounding alone separates FP32 and FP64 runs by ~1e-4."""
    from .golden.make_golden import TRAJ_ITERS, traj_scene, traj_sphere_path
    g = np.load(os.path.join(GOLDEN, "ref_traj.npz"))
    m, fixed = traj_scene()
    o = Oracle(m, mg.default_params(mg.SOLVER_REFERENCE_JACOBI, iterations=TRAJ_ITERS))
    o.set_fixed(fixed)
    path = traj_sphere_path()
    keep = list(g["frames"])
    tol = 5e-5 * m.bbox_diagonal()
    for f in range(path.shape[0]):
        o.set_spheres(path[f, :3][None], [path[f, 3]])
        o.step()
        if f in keep:
            k = keep.index(f)
            err = np.abs(o.positions() - g["positions"][k]).max()
            assert err < tol, (f, err, tol)
            assert np.array_equal(o.contact_flags(), g["flags"][k]), f


def test_reference_iteration_sensitivity(oracle_built):
    """Documents why the reference kind is pinned at 5e-5 x diag: a 1e-6 state
    perturbation grows to > 1e-5 within ten frames of the reference iteration."""
    from .golden.make_golden import TRAJ_ITERS, traj_scene, traj_sphere_path
    m, fixed = traj_scene()
    path = traj_sphere_path()
    runs = []
    for pert in (0.0, 1e-6):
        o = Oracle(m, mg.default_params(mg.SOLVER_REFERENCE_JACOBI, iterations=TRAJ_ITERS))
        o.set_fixed(fixed)
        x = m.positions.astype(np.float64) + np.random.default_rng(0).normal(0, pert, m.positions.shape)
        x[fixed.astype(bool)] = m.positions[fixed.astype(bool)]
        o.set_state(x, None)
        for f in range(10):
            o.set_spheres(path[f, :3][None], [path[f, 3]])
            o.step()
        runs.append(o.positions())
    amp = np.abs(runs[0] - runs[1]).max() / 1e-6
    assert amp > 10.0


def test_oracle_surface_normals_box():
    """UpdateTriNormal + AvgOutsideTetVertNormal restated: on a box every surface
    normal is a unit vector pointing outward, a face-interior vertex gets the
    face's axis, and interior vertices get zero."""
    from oracle.binding import surface_normals
    m = mg.box_mesh(3, 4, 5, (0.0, 0.0, 0.0), (3.0, 4.0, 5.0))
    mg.extract_surface(m)
    n = surface_normals(m.positions, m.tris)
    surf = np.unique(m.tris)
    inner = np.setdiff1d(np.arange(m.num_verts), surf)
    assert np.all(n[inner] == 0.0)
    assert np.allclose(np.linalg.norm(n[surf], axis=1), 1.0)
    assert np.all(np.einsum("ij,ij->i", n[surf], m.positions[surf] - m.positions.mean(0)) > 0)
    x = m.positions
    face = np.nonzero((x[:, 2] == 5.0) & (x[:, 0] == 1.0) & (x[:, 1] == 2.0))[0]
    assert np.allclose(n[face], [[0.0, 0.0, 1.0]])


def test_oracle_two_level_binding_and_steps():
    """The two-level restatement binds the nested golden meshes (every fine vertex
    in a coarse tet, every coarse vertex in a fine tet) and steps finitely."""
    from oracle.binding import OracleTwoLevel
    from .golden.make_golden import mg2_scene, traj_sphere_path
    coarse, fine, cf, ff = mg2_scene()
    o = OracleTwoLevel(coarse, fine, mg.default_params(mg.SOLVER_REFERENCE_JACOBI))
    o.set_fixed(cf, ff)
    path = traj_sphere_path(5)
    for f in range(5):
        o.set_spheres(path[f, :3][None], [path[f, 3]])
        o.step()
    for lvl in (0, 1):
        assert np.isfinite(o.positions(lvl)).all()
    # fixed vertices stay at rest on both levels (the transfers rewrite them, as in the
    # reference's updatePointInTet, so to rounding)
    assert np.abs(o.positions(0)[ff == 1] - fine.positions[ff == 1]).max() < 1e-12
    assert np.abs(o.positions(1)[cf == 1] - coarse.positions[cf == 1]).max() < 1e-12
