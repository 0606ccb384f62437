"""The reference's two-level schedule (PDSolver_MG) on the GPU against the FP64
oracle's restatement and against the reference's own GPU frames."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import OracleTwoLevel

from .golden.make_golden import MG2_FRAMES, MG2_KEEP, mg2_scene, traj_sphere_path

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_mg2_traj.npz")


def _run(obj, coarse_fixed, fine_fixed, frames, keep=None):
    obj.set_fixed(coarse_fixed, fine_fixed)
    path = traj_sphere_path(frames)
    out = {}
    for f in range(frames):
        obj.set_spheres(path[f, :3][None], [path[f, 3]])
        obj.step()
        if keep is None or f in keep:
            out[f] = (obj.positions(0).astype(np.float64), obj.positions(1).astype(np.float64))
    return out


def test_two_level_matches_oracle(lib, oracle_built):
    coarse, fine, cf, ff = mg2_scene()
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    t = mg.TwoLevel(coarse, fine, p)
    o = OracleTwoLevel(coarse, fine, p)
    got = _run(t, cf, ff, MG2_FRAMES, set(MG2_KEEP))
    want = _run(o, cf, ff, MG2_FRAMES, set(MG2_KEEP))
    diag = fine.bbox_diagonal()
    for f in MG2_KEEP:
        ef = np.abs(got[f][0] - want[f][0]).max()
        ec = np.abs(got[f][1] - want[f][1]).max()
        # reference-kind tolerance: FP32 vs FP64 of an iteration that amplifies perturbations
        assert ef < 5e-5 * diag and ec < 5e-5 * diag, (f, ef, ec)
    fl = t.levels[1].contact_flags()
    assert fl.sum() > 0                      # the coarse level saw triangle contacts
    t.close()


def test_two_level_matches_reference_gpu(lib):
    if not os.path.exists(GOLDEN):
        pytest.skip("ref_mg2_traj.npz not generated")
    g = np.load(GOLDEN)
    coarse, fine, cf, ff = mg2_scene()
    p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI)
    t = mg.TwoLevel(coarse, fine, p)
    keep = [int(f) for f in g["frames"]]
    got = _run(t, cf, ff, MG2_FRAMES, set(keep))
    diag = fine.bbox_diagonal()
    noise = float(g["rerun_maxdiff"].max())
    for k, f in enumerate(keep):
        ef = np.abs(got[f][0] - g["fine"][k]).max()
        ec = np.abs(got[f][1] - g["coarse"][k]).max()
        assert ef < 5e-5 * diag + noise and ec < 5e-5 * diag + noise, (f, ef, ec, noise)
    t.close()
