"""Scaled configurations against the FP64 oracle over their tool paths.

* Config 3 (batched uneven bodies): a seeded subset of the 256-body batch -- the
  first 8 bodies the benchmark generates from seed 11 (n x 10n x n hexes, n in
  {2..8}, per-body E, nu and capsule) -- advanced in one batch for 200 frames,
  each body against its own oracle.
* Config 4 (the organ-like blob): the learned smoother with mixed precision at
  1 V-cycle per PD iteration and 1+1 coarse sweeps (the committed network)
  against the oracle converging its global step (6 V-cycles per PD iteration),
  100 frames of the tool path.
Tolerance: max vertex distance <= 1e-5 x bbox diagonal; contact vertex index
sets bit-exact."""
import os

import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200 import sweeps
from oracle.binding import Oracle

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_config3_batch_subset_200_frames(lib, oracle_built):
    import bench
    meshes, params, fixeds, tool, _, mats = bench.make_workload("batch", mg)
    k = 8
    meshes, params, fixeds, mats = meshes[:k], params[:k], fixeds[:k], mats[:k]
    assert len({m.num_tets for m in meshes}) >= 4   # uneven sizes
    s = mg.Solver(meshes, params)
    orc = []
    for b in range(k):
        s.set_fixed(fixeds[b], body=b)
        s.set_material(*mats[b], body=b)
        o = Oracle(meshes[b], params[b])
        o.set_fixed(fixeds[b])
        o.set_material(*mats[b])
        orc.append(o)
    worst = [0.0] * k
    touched = 0
    for f in range(200):
        a, c, r = tool(f)
        s.set_capsules(a[:k], c[:k], r[:k])
        s.step()
        for b, o in enumerate(orc):
            o.set_capsule(a[b], c[b], float(r[b]))
            o.step()
        if f % 10 == 9:
            for b, o in enumerate(orc):
                cg, co = np.nonzero(s.contact_flags(b))[0], np.nonzero(o.contact_flags())[0]
                assert np.array_equal(cg, co), (f, b, np.setxor1d(cg, co))
                touched += len(co)
                d = sweeps.max_vertex_error(s.positions(b), o.positions()) / meshes[b].bbox_diagonal()
                worst[b] = max(worst[b], d)
    print("config 3 subset: max vertex distance / diag per body", worst, "contacts seen", touched)
    assert touched > 0
    assert max(worst) <= 1e-5, worst
    s.close()


def test_config4_blob_learned_mixed_100_frames(lib, oracle_built):
    from multigridsoftbody_b200.learned import MLP, blob_scene, blob_tool_path
    m, fixed, p = blob_scene(precision=mg.PRECISION_MIXED, refinement_passes=1)
    p.pre_sweeps, p.post_sweeps = 1, 1
    net = MLP(device=0, seed=0)
    net.params = np.load(os.path.join(ROOT, "tests", "golden", "beam_smoother.npy"))
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    s.set_learned_smoother(net, 0.5)
    o = Oracle(m, sweeps.variant_params(p, (2, 2), 6, True))
    o.set_fixed(fixed)
    path = blob_tool_path(100, seed=1)
    xor, touched = 0, 0
    for f, (a, b) in enumerate(path):
        for x in (s, o):
            x.set_capsule(a, b, 0.3)
            x.step()
        cg, co = np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0]
        xor += len(np.setxor1d(cg, co))
        touched += len(co)
    err = sweeps.max_vertex_error(s.positions_f64(), o.positions()) / m.bbox_diagonal()
    cycles, failed = s.learned_stats()
    print(f"config 4 blob: max vertex distance / diag {err:.3e}, contact XOR {xor} of {touched}, "
          f"learned checks {cycles} failed {failed}")
    assert touched > 0
    assert err <= 1e-5, err
    assert xor == 0
    assert cycles == 100 * p.iterations and failed <= cycles // 10
    s.close()
