"""The uniform-grid broad phase of the tool contact against the all-vertex
test: the same candidates reach the same narrow-phase test, so contact sets,
stiffness and every frame are the same bit for bit (FP32 graph and eager,
mixed precision, a batch of uneven bodies, a tool that leaves the grid)."""
import numpy as np
import pytest

import multigridsoftbody_b200 as mg

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu


def _run(meshes, fixeds, p, tools, broad):
    s = mg.Solver(meshes, p)
    for b, f in enumerate(fixeds):
        s.set_fixed(f, body=b)
    s.set_broad_phase(broad)
    flags = []
    for frame in tools:
        for b, (a, c, r) in enumerate(frame):
            s.set_capsule(a, c, r, body=b)
        s.step()
        flags.append([s.contact_flags(b).copy() for b in range(len(fixeds))])
    x = [s.positions(b) for b in range(len(fixeds))]
    s.close()
    return flags, x


def _assert_same(meshes, fixeds, p, tools):
    fa, xa = _run(meshes, fixeds, p, tools, False)
    fb, xb = _run(meshes, fixeds, p, tools, True)
    touched = 0
    for f_all, f_bp in zip(fa, fb):
        for u, v in zip(f_all, f_bp):
            assert np.array_equal(u, v)
            touched += int(u.sum())
    for u, v in zip(xa, xb):
        assert np.array_equal(u, v)
    return touched


@pytest.mark.parametrize("precision,graph", [(mg.PRECISION_FP32, 1), (mg.PRECISION_FP32, 0), (mg.PRECISION_MIXED, 1)])
def test_broad_phase_equals_all_vertex_test(lib, precision, graph):
    m, fixed = beam(6, 60, 6)
    p = mg_params(levels=3, gravity=(0, 0, 0), precision=precision, refinement_passes=1, use_graph=graph)
    path = capsule_path(30, start=(0.0, 0.0, 1.35))
    tools = [[(a, b, 0.3)] for a, b in path]
    assert _assert_same([m], [fixed], p, tools) > 0


def test_broad_phase_batch_and_tool_outside_grid(lib):
    """Bodies of different sizes, each with its own capsule; body 1's capsule
    starts far outside its grid (clamped query) and body 2 has no tool."""
    m0, f0 = beam(4, 40, 4)
    m1, f1 = beam(3, 20, 5, half_len=5.0)
    m2, f2 = beam(2, 10, 2, half_len=2.5)
    p = mg_params(levels=3, gravity=(0, 0, 0))
    path0 = capsule_path(20, start=(0.0, 0.0, 1.3))
    path1 = capsule_path(20, start=(0.0, 0.0, 40.0), dz=-2.0)   # sweeps in from z = 40
    zero = np.zeros(3, np.float32)
    tools = [[(a0, b0, 0.3), (a1, b1, 0.4), (zero, zero, 0.0)] for (a0, b0), (a1, b1) in zip(path0, path1)]
    assert _assert_same([m0, m1, m2], [f0, f1, f2], p, tools) > 0


def test_broad_phase_toggle_mid_run(lib):
    """Switching the broad phase on and off between frames keeps the frames
    equal to the all-vertex run."""
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, gravity=(0, 0, 0))
    path = capsule_path(16, start=(0.0, 0.0, 1.3))
    ref = mg.Solver(m, p)
    s = mg.Solver(m, p)
    for sv in (ref, s):
        sv.set_fixed(fixed)
    for f, (a, b) in enumerate(path):
        if f in (4, 8, 12):
            s.set_broad_phase(f != 8)
        for sv in (ref, s):
            sv.set_capsule(a, b, 0.3)
            sv.step()
        assert np.array_equal(ref.contact_flags(), s.contact_flags())
    assert np.array_equal(ref.positions(), s.positions())
    ref.close()
    s.close()
