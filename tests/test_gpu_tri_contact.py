"""Capsule against the surface triangles (mgsb_set_surface_contact) on the GPU
against the FP64 oracle's restatement: a capsule that enters coarse faces
between their vertices is found only by the triangle test; the contact vertex
sets are bit-exact every frame and the positions stay within 1e-5 x bbox
diagonal, in the FP32 and the mixed-precision kinds, and a batch gives the
same bits as its bodies run alone."""
import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle

from .common import beam, mg_params

pytestmark = pytest.mark.gpu


def _path(frames, y=0.5, z0=1.15, dz=-0.02):
    """Capsule along x (segment -3..3), radius 0.2, midway between two vertex rows of a coarse beam,
    sinking 0.02 per frame: its first frame touches the top faces but no vertex; the pushed surface
    then moves away and the capsule catches up with it again."""
    return [(np.array([-3.0, y, z0 + dz * f], np.float32), np.array([3.0, y, z0 + dz * f], np.float32))
            for f in range(frames)]


def _run_pair(precision, frames=40):
    m, fixed = beam(2, 20, 2)
    p = mg_params(levels=2, gravity=(0.0, 0.0, 0.0), precision=precision,
                  refinement_passes=2 if precision == mg.PRECISION_MIXED else 1)
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    s.set_surface_contact(True)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    o.set_surface_contact(True)
    tol = 1e-5 * m.bbox_diagonal()
    worst, ncontact = 0.0, []
    for f, (a, b) in enumerate(_path(frames)):
        for x in (s, o):
            x.set_capsule(a, b, 0.2)
            x.step()
        cg, co = np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0]
        assert np.array_equal(cg, co), (f, np.setxor1d(cg, co))
        ncontact.append(len(co))
        xs = s.positions_f64() if precision == mg.PRECISION_MIXED else s.positions()
        worst = max(worst, float(np.abs(xs - o.positions()).max()))
    s.close()
    return worst, tol, ncontact


@pytest.mark.parametrize("precision", [mg.PRECISION_FP32, mg.PRECISION_MIXED])
def test_triangle_contact_matches_oracle(lib, oracle_built, precision):
    worst, tol, ncontact = _run_pair(precision)
    print(f"triangle contact, precision {precision}: contacts per frame {ncontact}, max error {worst:.3e} m")
    assert ncontact[0] > 0 and sum(1 for c in ncontact if c) >= 5, ncontact
    assert worst < tol, (worst, tol)


def test_vertex_test_misses_what_triangles_find(lib):
    m, fixed = beam(2, 20, 2)
    p = mg_params(levels=2, gravity=(0.0, 0.0, 0.0))
    counts = {}
    for tri in (False, True):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_surface_contact(tri)
        a, b = _path(1)[0]
        s.set_capsule(a, b, 0.2)
        s.step()
        counts[tri] = int(s.contact_flags().sum())
        s.close()
    assert counts[False] == 0 and counts[True] > 0


def test_triangle_contact_batch_equals_single_bodies(lib):
    meshes, fixeds = [], []
    for n in (2, 3):
        m, fx = beam(n, 10 * n, n, half_len=2.5 * n)
        meshes.append(m)
        fixeds.append(fx)
    p = mg_params(levels=2, gravity=(0.0, 0.0, 0.0))
    batch = mg.Solver(meshes, [p, p])
    singles = [mg.Solver(m, p) for m in meshes]
    for i, fx in enumerate(fixeds):
        batch.set_fixed(fx, body=i)
        singles[i].set_fixed(fx)
        singles[i].set_surface_contact(True)
    batch.set_surface_contact(True)
    touched = 0
    for f in range(15):
        for i in range(2):
            a = np.array([-3.0, 0.3 * i + 0.25, 1.12 - 0.004 * f], np.float32)
            b = np.array([3.0, 0.3 * i + 0.25, 1.12 - 0.004 * f], np.float32)
            batch.set_capsule(a, b, 0.2, body=i)
            singles[i].set_capsule(a, b, 0.2)
            singles[i].step()
        batch.step()
        for i in range(2):
            assert np.array_equal(batch.positions(i), singles[i].positions())
            assert np.array_equal(batch.contact_flags(i), singles[i].contact_flags())
            touched += int(batch.contact_flags(i).sum())
    assert touched > 0
    for x in [batch] + singles:
        x.close()


def test_triangle_contact_and_broad_phase_exclusive(lib):
    m, fixed = beam(2, 20, 2)
    s = mg.Solver(m, mg_params(levels=2))
    s.set_fixed(fixed)
    s.set_surface_contact(True)
    with pytest.raises(mg.MgsbError):
        s.set_broad_phase(True)
    s.set_surface_contact(False)
    s.set_broad_phase(True)
    with pytest.raises(mg.MgsbError):
        s.set_surface_contact(True)
    s.close()
