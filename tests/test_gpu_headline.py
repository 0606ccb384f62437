"""The headline configuration pinned to the FP64 oracle.

The benchmark's metric compares the learned smoother with mixed precision and
the plain FP32 multigrid on the 12x120x12-hex beam (20,449 vertices, 103,680
tets, 4 levels, gravity off, top face fixed) at max vertex error <= 1e-5 x bbox
diagonal after 100 frames, the error taken against the converged frame.  The
tool is the config-1 capsule (r 0.3, segment length 8 along x) moving -z by
0.02 per frame plus N(0, 0.005^2) jitter (seed 1), on two paths: as
configured from z = 3, and started at z = 1.5 so that it is in contact from
frame ~10 (the benchmark's timed path).

Here, over both paths, the FP64 oracle converges each frame's global steps
(6 V-cycles with 2+2 sweeps per PD iteration) and runs beside
* the GPU solver the benchmark measures its error bar against (mixed
  precision, 6 V-cycles per PD iteration, plain smoother): it must be the
  oracle's frame to well below the bar, with the same contact sets;
* the learned smoother with mixed precision (the committed network) at 2 and
  at 1 V-cycles per PD iteration, 1+1 coarse sweeps, and the 2-cycle form in
  the shape the benchmark's autotuner picks (levels 2-3 as the dense coarse
  operator).  The 2-cycle forms must be within the bar; the 1-cycle form's
  error is printed (it is within the bar on some paths only, so it is not the
  headline form).
The reference iteration these frames restate is PDSolver::Step
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


@pytest.mark.parametrize("start_z", [3.0, 1.5])
def test_headline_vs_fp64_oracle_100_frames(lib, oracle_built, start_z):
    from multigridsoftbody_b200.learned import MLP
    m, fixed = beam(12, 120, 12)
    base = mg.default_params(mg.SOLVER_MULTIGRID, levels=4, iterations=10, gravity=(0.0, 0.0, 0.0),
                             precision=mg.PRECISION_MIXED, refinement_passes=1)
    net = MLP(device=0, seed=0)
    net.params = np.load(os.path.join(ROOT, "tests", "golden", "beam_smoother.npy"))
    solvers = {"converged": mg.Solver(m, sweeps.variant_params(base, (2, 2), 6, True))}
    for passes in (2, 1):
        s = mg.Solver(m, sweeps.variant_params(base, (1, 1), passes, True))
        s.set_learned_smoother(net, 0.5)
        solvers[f"learned_{passes}pass"] = s
    # the benchmark's autotuned shape: level 1 grid-wide, levels 2-3 as the dense coarse operator
    s = mg.Solver(m, sweeps.variant_params(base, (1, 1), 2, True))
    s.set_learned_smoother(net, 0.5)
    s.set_coarse_split(2)
    s.set_coarse_dense(True)
    solvers["learned_2pass_dense"] = s
    o = Oracle(m, sweeps.variant_params(base, (2, 2), 6, True))
    for x in list(solvers.values()) + [o]:
        x.set_fixed(fixed)
    path = capsule_path(FRAMES, start=(0.0, 0.0, start_z), seed=1)
    xor = dict.fromkeys(solvers, 0)
    touched = 0
    for a, b in path:
        for x in list(solvers.values()) + [o]:
            x.set_capsule(a, b, 0.3)
            x.step()
        co = np.nonzero(o.contact_flags())[0]
        touched += len(co)
        for k, s in solvers.items():
            xor[k] += len(np.setxor1d(np.nonzero(s.contact_flags())[0], co))
    diag = m.bbox_diagonal()
    xo = o.positions()
    err = {k: sweeps.max_vertex_error(s.positions_f64(), xo) / diag for k, s in solvers.items()}
    stats = {k: s.learned_stats() for k, s in solvers.items() if k.startswith("learned")}
    print(f"start z={start_z}, {FRAMES} frames: error / diag {err}; contact XOR vs oracle {xor} of {touched}; "
          f"learned checks (cycles, failed) {stats}")
    assert touched > 0
    # the benchmark's error reference is the oracle's frame to well below the bar
    assert err["converged"] <= 1e-6, err
    assert xor["converged"] == 0
    # the headline learned form meets the bar
    for k in ("learned_2pass", "learned_2pass_dense"):
        assert err[k] <= 1e-5, err
        assert xor[k] <= touched // 1000, xor
    for s in solvers.values():
        s.close()
    net.close()
