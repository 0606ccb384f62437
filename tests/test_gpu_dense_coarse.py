"""The dense coarse operator (mgsb_set_coarse_dense): the V-cycle of the levels
from the coarse split down, formed once per frame as a matrix and applied as
one restriction + one dense product, gives the same frames as the cluster or
one-CTA kernels up to rounding, and matches the FP64 oracle within 1e-5 x bbox
diagonal with bit-exact contact sets (FP32 and mixed precision, plain and
learned cycles)."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200.sweeps import max_vertex_error
from oracle.binding import Oracle

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(m, fixed, p, split, dense, frames, net=None):
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    if net is not None:
        s.set_learned_smoother(net, 0.5)
    s.set_coarse_split(split)
    s.set_coarse_dense(dense)
    flags = []
    for a, b in capsule_path(frames, start=(0.0, 0.0, 1.4)):
        s.set_capsule(a, b, 0.3)
        s.step()
        flags.append(np.nonzero(s.contact_flags())[0])
    assert s.coarse_dense() == dense
    x = s.positions_f64() if p.precision == mg.PRECISION_MIXED else s.positions().astype(np.float64)
    s.close()
    return x, flags


@pytest.mark.parametrize("precision,split", [(mg.PRECISION_FP32, 1), (mg.PRECISION_FP32, 2),
                                             (mg.PRECISION_MIXED, 1), (mg.PRECISION_MIXED, 2)])
def test_dense_operator_matches_kernel_and_oracle(lib, oracle_built, precision, split):
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, gravity=(0.0, 0.0, 0.0), precision=precision,
                  refinement_passes=2 if precision == mg.PRECISION_MIXED else 1)
    frames = 30
    xk, fk = _run(m, fixed, p, split, False, frames)
    xd, fd = _run(m, fixed, p, split, True, frames)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    for a, b in capsule_path(frames, start=(0.0, 0.0, 1.4)):
        o.set_capsule(a, b, 0.3)
        o.step()
    diag = m.bbox_diagonal()
    assert max_vertex_error(xd, xk) / diag < 1e-6
    assert max_vertex_error(xd, o.positions()) / diag < 1e-5
    assert all(np.array_equal(u, v) for u, v in zip(fd, fk))
    assert np.array_equal(fd[-1], np.nonzero(o.contact_flags())[0]) and len(fd[-1]) > 0


@pytest.mark.parametrize("split", [2, 3])
def test_dense_operator_config1_learned(lib, split):
    """The headline's beam (levels 2-3 as a 496 x 496 operator, or the 144 x 144 coarsest inverse
    alone) with the learned smoother and mixed precision: the same frames as the cluster kernel up
    to rounding, the same contact sets."""
    from multigridsoftbody_b200.learned import MLP
    m, fixed = beam(12, 120, 12)
    p = mg_params(levels=4, gravity=(0.0, 0.0, 0.0), precision=mg.PRECISION_MIXED, refinement_passes=2,
                  pre_sweeps=1, post_sweeps=1)
    net = MLP(device=0, seed=0)
    net.params = np.load(os.path.join(ROOT, "tests", "golden", "beam_smoother.npy"))
    xk, fk = _run(m, fixed, p, split, False, 20, net)
    xd, fd = _run(m, fixed, p, split, True, 20, net)
    assert max_vertex_error(xd, xk) / m.bbox_diagonal() < 1e-6
    assert all(np.array_equal(u, v) for u, v in zip(fd, fk))


def test_dense_operator_refused_for_a_batch(lib):
    meshes, fixeds = [], []
    for n in (2, 3):
        mm, fx = beam(n, 10 * n, n, half_len=2.5 * n)
        meshes.append(mm)
        fixeds.append(fx)
    p = mg_params(levels=3)
    s = mg.Solver(meshes, [p, p])
    with pytest.raises(mg.MgsbError):
        s.set_coarse_dense(True)
    s.close()


def test_dense_operator_refused_above_its_row_limit(lib):
    """Config 1's level 1 has 2,989 rows, above the operator's 1,024: the dense operator is refused at
    split 1 and the solver keeps stepping with the kernel path; at split 2 (496 rows) it is accepted."""
    m, fixed = beam(12, 120, 12)
    s = mg.Solver(m, mg_params(levels=4, gravity=(0.0, 0.0, 0.0)))
    s.set_fixed(fixed)
    assert s.body_level_size(0, 1) > 1024 >= s.body_level_size(0, 2)
    s.set_coarse_split(1)
    with pytest.raises(mg.MgsbError):
        s.set_coarse_dense(True)
    assert not s.coarse_dense()
    s.step()
    s.set_coarse_split(2)
    s.set_coarse_dense(True)
    assert s.coarse_dense()
    s.step()
    assert np.isfinite(s.positions()).all()
    s.close()
