"""Multigrid PD frame on the GPU (FP32) vs the FP64 oracle running the same
configured algorithm.  Tolerance: max vertex error <= 1e-5 x bbox diagonal;
contact vertex index sets bit-exact."""
import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from oracle.binding import Oracle

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu


def _pair(m, fixed, p):
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    return s, o


def test_level_sizes_match_oracle(lib, oracle_built):
    m, fixed = beam(12, 120, 12)
    p = mg_params(levels=4, gravity=(0, 0, 0))
    s, o = _pair(m, fixed, p)
    for l in range(4):
        assert s.level_size(l) == o.level_size(l), l
    assert [s.level_size(l)[0] for l in range(4)] == [20449, 2989, 496, 144]
    s.close()


def test_config0_gravity_parity(lib, oracle_built):
    """Config 0 (4x40x4 hexes, 3 levels, gravity, fixed y=+10, 200 frames), GPU FP32 vs FP64."""
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3)
    s, o = _pair(m, fixed, p)
    tol = 1e-5 * m.bbox_diagonal()
    worst = 0.0
    for f in range(200):
        s.step()
        o.step()
        if f % 20 == 19:
            worst = max(worst, np.abs(s.positions() - o.positions()).max())
    assert worst < tol, (worst, tol)
    fx = fixed.astype(bool)
    assert np.array_equal(s.positions()[fx], m.positions[fx])
    s.close()


def _tool_run(m, fixed, p, frames, path, check_every=1):
    s, o = _pair(m, fixed, p)
    tol = 1e-5 * m.bbox_diagonal()
    worst = 0.0
    ncontact = 0
    mismatches = []
    for f in range(frames):
        a, b = path[f]
        for solver in (s, o):
            solver.set_capsule(a, b, 0.3)
            solver.step()
        if f % check_every == 0 or f == frames - 1:
            worst = max(worst, np.abs(s.positions() - o.positions()).max())
            cg = np.nonzero(s.contact_flags())[0]
            co = np.nonzero(o.contact_flags())[0]
            ncontact += len(co)
            if not np.array_equal(cg, co):
                mismatches.append((f, np.setxor1d(cg, co)))
    s.close()
    return worst, tol, ncontact, mismatches


def test_tool_contact_parity_small(lib, oracle_built):
    """Config-1 tool path on the 4x40x4 beam (3 levels, gravity off), 120 frames."""
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, gravity=(0, 0, 0))
    path = capsule_path(120, start=(0.0, 0.0, 1.6))
    worst, tol, ncontact, mism = _tool_run(m, fixed, p, 120, path)
    assert ncontact > 0
    assert not mism, mism
    assert worst < tol, (worst, tol)


@pytest.mark.slow
def test_config1_parity_100_frames(lib, oracle_built):
    """Config 1: 12x120x12 hexes (103,680 tets), 4 levels, capsule r=0.3 length 8 from (0,0,3),
    -0.02 z per frame + N(0, 0.005^2) jitter, 100 frames.  The capsule reaches the beam
    at frame ~85, so the run starts from z=1.9 to cover 100 frames of contact."""
    m, fixed = beam(12, 120, 12)
    p = mg_params(levels=4, gravity=(0, 0, 0))
    path = capsule_path(100, start=(0.0, 0.0, 1.5))
    worst, tol, ncontact, mism = _tool_run(m, fixed, p, 100, path, check_every=5)
    assert ncontact > 0
    assert not mism, mism
    assert worst < tol, (worst, tol)


def test_batch_equals_single_bodies(lib):
    """Bodies batched in one launch per phase give the same bits as separate solvers."""
    rng = np.random.default_rng(11)
    meshes, fixeds, params = [], [], []
    for n in (2, 3, 2):
        m, fx = beam(n, 10 * n, n, half_len=2.5 * n)
        meshes.append(m)
        fixeds.append(fx)
        params.append(mg_params(levels=3, gravity=(0, 0, 0)))
    batch = mg.Solver(meshes, params)
    singles = [mg.Solver(m, p) for m, p in zip(meshes, params)]
    E = [np.exp(rng.uniform(np.log(5e4), np.log(2e5), m.num_tets)).astype(np.float32) for m in meshes]
    for i, (m, fx) in enumerate(zip(meshes, fixeds)):
        batch.set_fixed(fx, body=i)
        batch.set_material(E[i], 0.3, body=i)
        singles[i].set_fixed(fx)
        singles[i].set_material(E[i], 0.3)
    for f in range(20):
        for i in range(3):
            a = np.array([-4.0, 0.1 * i, 1.1 - 0.01 * f], np.float32)
            b = np.array([4.0, 0.1 * i, 1.1 - 0.01 * f], np.float32)
            batch.set_capsule(a, b, 0.2, body=i)
            singles[i].set_capsule(a, b, 0.2)
        batch.step()
        for s in singles:
            s.step()
    for i in range(3):
        assert np.array_equal(batch.positions(i), singles[i].positions()), i
        assert np.array_equal(batch.contact_flags(i), singles[i].contact_flags()), i


def test_graph_equals_eager(lib):
    m, fixed = beam(4, 40, 4)
    sols = []
    for g in (1, 0):
        s = mg.Solver(m, mg_params(levels=3, use_graph=g))
        s.set_fixed(fixed)
        s.step(25)
        sols.append(s.positions())
    assert np.array_equal(sols[0], sols[1])


def test_checkpoint_resume_bitwise(lib):
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    s.step(10)
    x, v = s.positions(), s.velocities()
    s.step(5)
    a = s.positions()
    s.set_state(x, v)
    s.step(5)
    assert np.array_equal(s.positions(), a)


def test_divergence_reported(lib):
    """A non-finite state (injected on the host) surfaces as MGSB_DIVERGED, not a fault."""
    m, fixed = beam(2, 10, 2)
    s = mg.Solver(m, mg_params(levels=2))
    s.set_fixed(fixed)
    x = m.positions.copy()
    x[5, 1] = np.nan
    s.set_state(x, None)
    s.step()
    with pytest.raises(mg.MgsbError) as e:
        s.positions()
    assert e.value.status == 4


@pytest.mark.parametrize("shape", [(1, 256, 0), (4, 1024, 1), (16, 512, 0), (2, 512, 1)])
def test_kernel_shapes_match_oracle(lib, oracle_built, shape):
    """Every coarse-kernel shape (cluster size, block size, level-0 fusion) gives
    the oracle's result on the tool scene."""
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, gravity=(0, 0, 0))
    s, o = _pair(m, fixed, p)
    s.set_kernel_shape(*shape)
    path = capsule_path(40, start=(0.0, 0.0, 1.4))
    for f in range(40):
        for solver in (s, o):
            solver.set_capsule(*path[f], 0.3)
            solver.step()
    assert np.abs(s.positions() - o.positions()).max() < 1e-5 * m.bbox_diagonal()
    assert np.array_equal(np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0])
    info = s.level_info(0)
    assert (info["cluster"], info["block"], info["fuse_l0"]) == shape


def test_autotune_restores_state(lib, oracle_built):
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3)
    s, o = _pair(m, fixed, p)
    s.step(5)
    o.step(5)
    chosen = s.autotune(frames=2)
    assert chosen["cluster"] >= 1 and chosen["block"] in (256, 512, 1024)
    s.step(5)
    o.step(5)
    assert np.abs(s.positions() - o.positions()).max() < 1e-5 * m.bbox_diagonal()


def test_mixed_precision_matches_oracle(lib, oracle_built):
    """Mixed precision (FP64 state and outer residual, FP32 V-cycle correction,
    FP64 coarsest, 2 refinement passes) vs the FP64 oracle running 2 V-cycles
    per PD iteration; closer to the oracle than the all-FP32 form."""
    m, fixed = beam(4, 40, 4)
    path = capsule_path(60, start=(0.0, 0.0, 1.4))
    errs = {}
    for prec in (mg.PRECISION_FP32, mg.PRECISION_MIXED):
        p = mg_params(levels=3, precision=prec, refinement_passes=2)
        s, o = _pair(m, fixed, p)
        for f in range(60):
            for solver in (s, o):
                solver.set_capsule(*path[f], 0.3)
                solver.step()
        xo = o.positions()
        errs[prec] = np.abs(s.positions().astype(np.float64) - xo).max()
        if prec == mg.PRECISION_MIXED:
            x64 = s.positions_f64()
            errs["f64"] = np.abs(x64 - xo).max()
            assert np.array_equal(np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0])
        s.close()
    tol = 1e-5 * m.bbox_diagonal()
    assert errs[mg.PRECISION_MIXED] < tol and errs["f64"] < tol, errs
    assert errs["f64"] <= errs[mg.PRECISION_FP32], errs


@pytest.mark.slow
def test_config2_mixed_precision(lib, oracle_built):
    """Config 2: 24x240x24 hexes (829,440 tets), 5 levels, per-tet E log-uniform in
    [5e4, 2e5] (seed 7), mixed precision with 2 refinement passes, the config-1 tool
    path started in contact, 100 frames.  Contact sets bit-exact at every 10th frame
    through frame 100; max vertex distance <= 1e-5 x diag at every 10th frame through
    frame 50.  Later frames are sensitivity-limited, not precision-limited: the FP64
    oracle itself, with its initial positions perturbed by 1e-9 m, drifts 6.2e-6 m by
    frame 50 and 8.4e-5 m (0.42 of the bar) by frame 100 on this scene, so the
    100-frame distance is printed, not asserted."""
    from multigridsoftbody_b200.sweeps import max_vertex_error
    m, fixed = beam(24, 240, 24)
    rng = np.random.default_rng(7)
    E = np.exp(rng.uniform(np.log(5e4), np.log(2e5), m.num_tets)).astype(np.float32)
    p = mg_params(levels=5, gravity=(0, 0, 0), precision=mg.PRECISION_MIXED, refinement_passes=2)
    s, o = _pair(m, fixed, p)
    s.set_material(E, 0.3)
    o.set_material(E, 0.3)
    frames = 100
    path = capsule_path(frames, start=(0.0, 0.0, 1.25))
    tol = 1e-5 * m.bbox_diagonal()
    errs, touched = {}, 0
    for f in range(frames):
        for solver in (s, o):
            solver.set_capsule(*path[f], 0.3)
            solver.step()
        if f % 10 == 9:
            errs[f + 1] = max_vertex_error(s.positions_f64(), o.positions())
            cg, co = np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0]
            assert np.array_equal(cg, co), (f, np.setxor1d(cg, co))
            touched += len(co)
    print(f"config 2: max vertex distance (m) at every 10th frame {errs} (tolerance {tol:.3e}); {touched} contacts")
    assert max(e for f, e in errs.items() if f <= 50) < tol, (errs, tol)
    assert touched > 0
    s.close()


def test_coarsest_update_many_contacts(lib, oracle_built):
    """A capsule that swallows a cube puts every coarsest boundary vertex in
    contact (98 of 125, more than the low-rank update handles), so the coarsest
    inverse is refactorised; a short capsule pressed on the top face touches a
    strip and takes the low-rank (Woodbury) update.  Both agree with the oracle."""
    m = mg.box_mesh(16, 16, 16, (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    fixed = np.zeros(m.num_verts, np.uint8)
    for z, radius, frames in ((0.0, 1.9, 2), (1.25, 0.4, 6)):
        p = mg_params(levels=3, gravity=(0.0, 0.0, 0.0))
        s, o = _pair(m, fixed, p)
        assert s.level_size(2)[0] == 125
        a = np.array([-0.1, 0.0, z], np.float32)
        b = np.array([0.1, 0.0, z], np.float32)
        touched = 0
        for f in range(frames):
            for solver in (s, o):
                solver.set_capsule(a, b, radius)
                solver.step()
            touched += o.contact_flags().sum()
        assert touched > 0
        err = np.abs(s.positions() - o.positions()).max()
        assert err < 1e-5 * m.bbox_diagonal(), (radius, err)
        s.close()


@pytest.mark.parametrize("precision,graph", [(mg.PRECISION_FP32, 1), (mg.PRECISION_FP32, 0), (mg.PRECISION_MIXED, 1)])
def test_coarse_split_same_frames(lib, oracle_built, precision, graph):
    """Running the first coarse levels as grid-wide kernels instead of inside
    the cluster kernel keeps every row's arithmetic (same lanes, same order),
    so all splits give the same frames; the last split also matches the oracle."""
    m, fixed = beam(8, 80, 8)
    p = mg_params(levels=4, gravity=(0, 0, 0), precision=precision, refinement_passes=2, use_graph=graph)
    path = capsule_path(20, start=(0.0, 0.0, 1.3))
    runs = {}
    for split in (1, 2, 3):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_coarse_split(split)
        assert s.coarse_split() == split
        for a, b in path:
            s.set_capsule(a, b, 0.3)
            s.step()
        runs[split] = (s.positions_f64() if precision == mg.PRECISION_MIXED else s.positions().astype(np.float64),
                       np.nonzero(s.contact_flags())[0])
        s.close()
    diag = m.bbox_diagonal()
    for split in (2, 3):
        assert np.abs(runs[split][0] - runs[1][0]).max() <= 1e-6 * diag, split
        assert np.array_equal(runs[split][1], runs[1][1])
    o = Oracle(m, p)
    o.set_fixed(fixed)
    for a, b in path:
        o.set_capsule(a, b, 0.3)
        o.step()
    assert np.abs(runs[3][0] - o.positions()).max() < 1e-5 * diag
    assert np.array_equal(runs[3][1], np.nonzero(o.contact_flags())[0])


def test_coarse_split_default_by_size(lib):
    """By size: coarse levels above 1024 rows run grid-wide (config 2's levels
    1 and 2 have 20,449 and 2,989), smaller ones stay in the cluster kernel."""
    small = mg.Solver(beam(4, 40, 4)[0], mg_params(levels=3))
    assert small.coarse_split() == 1
    big = mg.Solver(beam(24, 240, 24)[0], mg_params(levels=5))
    assert big.level_size(2)[0] == 2989 and big.coarse_split() == 3
    with pytest.raises(mg.MgsbError):
        big.set_coarse_split(5)
    # one CTA cannot hold levels 1-4 (24,078 rows) in shared memory: a clear error, not a bad frame
    big.set_kernel_shape(1, 1024, 0)
    big.set_coarse_split(1)
    with pytest.raises(mg.MgsbError) as err:
        big.step()
    assert err.value.status == 6
    small.close()
    big.close()


@pytest.mark.parametrize("kind", ["fp32_graph", "fp32_eager", "mixed", "reference", "batch"])
def test_launch_overlap_bitwise(lib, kind):
    """Programmatic dependent launch only moves when a kernel's blocks are
    scheduled; each still waits for its predecessor, so frames are bitwise
    the same with it on and off."""
    m, fixed = beam(4, 40, 4)
    meshes, fixeds = m, [fixed]
    if kind == "reference":
        p = mg.default_params(mg.SOLVER_REFERENCE_JACOBI, iterations=10)
    elif kind == "mixed":
        p = mg_params(levels=3, precision=mg.PRECISION_MIXED, refinement_passes=2)
    else:
        p = mg_params(levels=3, use_graph=0 if kind == "fp32_eager" else 1)
    if kind == "batch":
        m1, f1 = beam(3, 20, 5, half_len=5.0)
        meshes, fixeds = [m, m1], [fixed, f1]
    path = capsule_path(12, start=(0.0, 0.0, 1.3))
    out = {}
    for on in (True, False):
        s = mg.Solver(meshes, p)
        for b, f in enumerate(fixeds):
            s.set_fixed(f, body=b)
        s.set_launch_overlap(on)
        for a, b in path:
            if kind == "reference":
                s.set_spheres(((a + b) / 2)[None], [0.6])
            else:
                s.set_capsule(a, b, 0.3)
            s.step()
        out[on] = [s.positions(b) for b in range(len(fixeds))]
        s.close()
    for x_on, x_off in zip(out[True], out[False]):
        assert np.array_equal(x_on, x_off)


@pytest.mark.parametrize("split", [1, 2, 3])
def test_one_cta_kernel_equals_cluster_kernel(lib, split):
    """A cluster of one CTA runs the one-CTA kernel (every owned level in
    shared memory, block barriers); it keeps the cluster kernel's lanes and
    summation order, so the frames are the same bit for bit."""
    m, fixed = beam(8, 80, 8)
    p = mg_params(levels=4, gravity=(0, 0, 0), use_graph=1)
    path = capsule_path(10, start=(0.0, 0.0, 1.3))
    out = {}
    for cluster in (1, 4):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_kernel_shape(cluster, 512, 0)
        s.set_coarse_split(split)
        for a, b in path:
            s.set_capsule(a, b, 0.3)
            s.step()
        assert s.level_info(0)["cluster"] == cluster
        out[cluster] = s.positions()
        s.close()
    assert np.array_equal(out[1], out[4])


@pytest.mark.parametrize("precision,split", [(mg.PRECISION_FP32, 2), (mg.PRECISION_FP32, 1), (mg.PRECISION_MIXED, 3)])
def test_fused_prolongation_same_vcycle(lib, oracle_built, precision, split):
    """Prolongation + first post-sweep as one kernel (from the descent's
    residual and OP = Off P) is the same V-cycle: the frames agree with the
    separate launches to rounding and both match the oracle."""
    m, fixed = beam(8, 80, 8)
    p = mg_params(levels=4, gravity=(0, 0, 0), precision=precision, refinement_passes=1)
    path = capsule_path(20, start=(0.0, 0.0, 1.3))
    runs = {}
    for fused in (True, False):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_coarse_split(split)
        s.set_fused_prolongation(fused)
        for a, b in path:
            s.set_capsule(a, b, 0.3)
            s.step()
        runs[fused] = (s.positions_f64() if precision == mg.PRECISION_MIXED else s.positions().astype(np.float64),
                       np.nonzero(s.contact_flags())[0])
        s.close()
    diag = m.bbox_diagonal()
    assert np.abs(runs[True][0] - runs[False][0]).max() < 1e-6 * diag
    assert np.array_equal(runs[True][1], runs[False][1])
    o = Oracle(m, p)
    o.set_fixed(fixed)
    for a, b in path:
        o.set_capsule(a, b, 0.3)
        o.step()
    assert np.abs(runs[True][0] - o.positions()).max() < 1e-5 * diag


@pytest.mark.parametrize("precision,split,learned", [(mg.PRECISION_FP32, 2, False), (mg.PRECISION_MIXED, 3, False),
                                                      (mg.PRECISION_MIXED, 2, True), (mg.PRECISION_FP32, 3, True)])
def test_fused_restriction_same_vcycle(lib, oracle_built, precision, split, learned):
    """Level 1's restriction straight from level 0 (R (b - D d) - RO d, RO = R Off0) and the
    level-0 residual rows formed by the fused prolongation are the same V-cycle: frames agree with
    the separate residual launch to rounding, contact sets are equal, one launch per V-cycle less,
    and the frames match the oracle (plain cycles)."""
    import os
    from multigridsoftbody_b200.learned import MLP
    m, fixed = beam(8, 80, 8)
    p = mg_params(levels=4, gravity=(0, 0, 0), precision=precision, refinement_passes=2)
    path = capsule_path(20, start=(0.0, 0.0, 1.3))
    net = None
    if learned:
        net = MLP(device=0, seed=0)
        net.params = np.load(os.path.join(os.path.dirname(__file__), "golden", "beam_smoother.npy"))
    runs, launches = {}, {}
    for fused in (True, False):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        if net is not None:
            s.set_learned_smoother(net, 0.5)
        s.set_coarse_split(split)
        s.set_fused_restriction(fused)
        for a, b in path:
            s.set_capsule(a, b, 0.3)
            s.step()
        runs[fused] = (s.positions_f64() if precision == mg.PRECISION_MIXED else s.positions().astype(np.float64),
                       np.nonzero(s.contact_flags())[0])
        launches[fused] = s.launches_per_frame()
        s.close()
    diag = m.bbox_diagonal()
    assert np.abs(runs[True][0] - runs[False][0]).max() < 1e-6 * diag
    assert np.array_equal(runs[True][1], runs[False][1])
    # one launch per V-cycle (the count covers the frame's main solve)
    assert launches[False] - launches[True] == p.iterations * p.refinement_passes, launches
    if not learned:
        o = Oracle(m, p)
        o.set_fixed(fixed)
        for a, b in path:
            o.set_capsule(a, b, 0.3)
            o.step()
        assert np.abs(runs[True][0] - o.positions()).max() < 1e-5 * diag


@pytest.mark.parametrize("precision", [mg.PRECISION_FP32, mg.PRECISION_MIXED])
def test_time_kernel_replays_without_changing_the_run(lib, precision):
    """Replay timing of every kernel of the frame: a positive time per launch,
    the launch count the profiled frame reports, and a run that continues
    bit for bit as if no replay had happened (the state is restored).  The
    broad-phase kernels are refused."""
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, gravity=(0, 0, 0), precision=precision, refinement_passes=1)
    path = capsule_path(10, start=(0.0, 0.0, 1.3))

    def make():
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_coarse_split(2)   # grid-wide level 1 and the cluster kernel
        s.set_broad_phase(True)
        return s

    probe = make()
    for a, b in path[:5]:
        probe.set_capsule(a, b, 0.3)
        probe.step()
    prof = probe.profile_frame()
    probe.close()
    assert "k_coarse_vcycle" in prof and "k_lvl_residual" in prof
    runs = []
    for timed in (False, True):
        s = make()
        for f, (a, b) in enumerate(path):
            s.set_capsule(a, b, 0.3)
            if timed and f == 5:
                for name, (_, count) in prof.items():
                    if name.startswith("k_bp_"):
                        with pytest.raises(mg.MgsbError):
                            s.time_kernel(name, 4)
                        continue
                    us, k = s.time_kernel(name, 4)
                    assert k == count and us > 0.0, (name, us, k, count)
            s.step()
        runs.append((s.positions(), s.contact_flags().copy()))
        s.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_frame_readback_equals_the_single_readbacks(lib):
    """mgsb_get_frame (positions + contact flags, one synchronisation) returns what the two single
    readbacks return, for a batch of bodies, into caller-owned arrays."""
    meshes, fixeds = [], []
    for n in (2, 3):
        m, fx = beam(n, 10 * n, n, half_len=2.5 * n)
        meshes.append(m)
        fixeds.append(fx)
    p = mg_params(levels=3, gravity=(0, 0, 0))
    s = mg.Solver(meshes, [p, p])
    for b, fx in enumerate(fixeds):
        s.set_fixed(fx, body=b)
    for a, b in capsule_path(12, start=(0.0, 0.0, 1.2)):
        s.set_capsules(np.stack([a, a]), np.stack([b, b]), np.array([0.3, 0.3], np.float32))
        s.step()
    nv = sum(m.num_verts for m in meshes)
    pos, flags = np.zeros((nv, 3), np.float32), np.zeros(nv, np.int32)
    out = s.frame(pos, flags)
    assert out[0] is pos and out[1] is flags
    assert np.array_equal(pos, s.all_positions())
    assert np.array_equal(flags, s.all_contact_flags()) and flags.sum() > 0
    with pytest.raises(ValueError):
        s.frame(np.zeros((nv, 3), np.float64), flags)
    # zero-copy: views of the pinned readback buffer, the same values
    pv, fv = s.frame_view()
    assert pv.shape == (nv, 3) and fv.shape == (nv,)
    assert np.array_equal(pv, pos) and np.array_equal(fv, flags)
    s.close()
