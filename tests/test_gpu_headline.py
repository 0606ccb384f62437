"""The headline configuration pinned to the FP64 oracle.

The benchmark's metric is the learned smoother with mixed precision at one
V-cycle per PD iteration and 1+1 coarse sweeps on the 12x120x12-hex beam
(20,449 vertices, 103,680 tets, 4 levels, gravity off, top face fixed), with
the capsule (r 0.3, segment length 8 along x) starting 0.3 above the beam and
moving -z by 0.02 per frame plus N(0, 0.005^2) jitter (seed 1), and its error
bar is max vertex error <= 1e-5 x bbox diagonal after 100 frames.  Here that
solver (the committed network, tests/golden/beam_smoother.npy) runs those 100
frames beside the FP64 oracle converging the same frames' global steps
(6 V-cycles with 2+2 sweeps per PD iteration: the exact PD frame to ~1e-8 of
the motion), and beside the GPU solver the benchmark measures its error bar
against (mixed precision, 6 V-cycles per PD iteration, plain smoother).  The
reference iteration these frames restate is PDSolver::Step
(PDSolver.cpp:243-293).  Max vertex error is the largest Euclidean distance of
a vertex."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200 import sweeps
from oracle.binding import Oracle

from .common import beam, capsule_path

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FRAMES = 100


def test_headline_learned_mixed_vs_fp64_oracle_100_frames(lib, oracle_built):
    from multigridsoftbody_b200.learned import MLP
    m, fixed = beam(12, 120, 12)
    base = mg.default_params(mg.SOLVER_MULTIGRID, levels=4, iterations=10, gravity=(0.0, 0.0, 0.0),
                             precision=mg.PRECISION_MIXED, refinement_passes=1)
    learned_p = sweeps.variant_params(base, (1, 1), 1, True)
    conv_p = sweeps.variant_params(base, (2, 2), 6, True)
    net = MLP(device=0, seed=0)
    net.params = np.load(os.path.join(ROOT, "tests", "golden", "beam_smoother.npy"))
    s = mg.Solver(m, learned_p)
    s.set_learned_smoother(net, 0.5)
    g = mg.Solver(m, conv_p)
    o = Oracle(m, conv_p)
    for x in (s, g, o):
        x.set_fixed(fixed)
    path = capsule_path(FRAMES, start=(0.0, 0.0, 1.5), seed=1)
    xor_learned = xor_conv = touched = 0
    for f, (a, b) in enumerate(path):
        for x in (s, g, o):
            x.set_capsule(a, b, 0.3)
            x.step()
        co = np.nonzero(o.contact_flags())[0]
        xor_learned += len(np.setxor1d(np.nonzero(s.contact_flags())[0], co))
        xor_conv += len(np.setxor1d(np.nonzero(g.contact_flags())[0], co))
        touched += len(co)
    diag = m.bbox_diagonal()
    xo = o.positions()
    err_learned = sweeps.max_vertex_error(s.positions_f64(), xo) / diag
    err_conv = sweeps.max_vertex_error(g.positions_f64(), xo) / diag
    cycles, failed = s.learned_stats()
    print(f"headline after {FRAMES} frames: learned+mixed {err_learned:.3e} x diag, GPU converged reference "
          f"{err_conv:.3e} x diag; contact XOR vs oracle: learned {xor_learned}, converged {xor_conv} "
          f"(of {touched} contacts); learned checks {cycles}, failed {failed}")
    assert touched > 0
    assert err_learned <= 1e-5, err_learned
    # the benchmark's error reference is the oracle's frame to well below the bar
    assert err_conv <= 1e-7, err_conv
    assert xor_conv == 0
    assert xor_learned <= touched // 1000, (xor_learned, touched)
    for x in (s, g):
        x.close()
