"""The learned smoother inside the V-cycle: training pairs from the plain
solver, training on the GPU, the gain over plain sweeps at equal sweep count,
the residual guard with its plain fallback (eager and in a CUDA graph), and
parity of the learned mixed-precision solver with the FP64 oracle."""
import numpy as np
import pytest

import multigridsoftbody_b200 as mg
from multigridsoftbody_b200.learned import MLP, NUM_PARAMS
from oracle.binding import Oracle

from .common import beam, capsule_path, mg_params

pytestmark = pytest.mark.gpu


def _train_on_beam(frames=24, steps=1500, seed=0):
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    xs, ts = [], []
    for f, (a, b) in enumerate(capsule_path(frames, start=(0.0, 0.0, 1.3), seed=seed + 3)):
        s.set_capsule(a, b, 0.3)
        s.step()
        if f % 4 == 3:
            x, t = s.smoother_pairs(4)
            xs.append(x)
            ts.append(t)
    s.close()
    x, t = np.concatenate(xs), np.concatenate(ts)
    net = MLP(seed=seed)
    losses = net.train(x, t, steps=steps, batch=2048, lr=2e-3, seed=seed + 1)
    return net, x, t, losses


@pytest.fixture(scope="module")
def trained():
    return _train_on_beam()


def test_pairs_and_training(lib, trained):
    net, x, t, losses = trained
    assert x.shape[1] == 9 and t.shape[1] == 3 and x.shape[0] == t.shape[0] > 1000
    assert np.isfinite(x).all() and np.isfinite(t).all()
    assert losses[-100:].mean() < 0.05 * losses[:10].mean(), (losses[:10].mean(), losses[-100:].mean())


def test_learned_sweep_gains_over_plain(lib, trained):
    """Ablation at equal sweep count: one learned sweep before and after the
    coarse correction against one Jacobi sweep each side (and, for scale,
    the configured two)."""
    net = trained[0]
    m, fixed = beam(4, 40, 4)
    s = mg.Solver(m, mg_params(levels=3))
    s.set_fixed(fixed)
    s.set_learned_smoother(net, 0.5)
    facs = {0: [], 1: [], 2: []}
    for f, (a, b) in enumerate(capsule_path(30, start=(0.0, 0.0, 1.3), seed=42)):
        s.set_capsule(a, b, 0.3)
        s.step()
        if f % 10 == 9:
            for mode in facs:
                r = s.vcycle_residuals(4, mode)
                facs[mode].append((r[-1] / r[0]) ** 0.25)
    plain22, plain11, learned = (np.mean(facs[k]) for k in (0, 1, 2))
    assert learned < 0.7 * plain11, (plain22, plain11, learned)
    assert learned < 1.5 * plain22, (plain22, plain11, learned)
    v, fb = s.learned_stats()
    assert v > 0 and fb <= v // 10, (v, fb)
    s.close()


@pytest.mark.parametrize("graph,split", [(1, 1), (0, 1), (1, 2), (0, 2)])
def test_guard_falls_back_to_plain(lib, graph, split):
    """A network with wild weights fails the residual check on every V-cycle;
    each frame's solve is then repeated with the plain V-cycle, so every
    frame equals the plain solver's bit for bit (also with level 1 run as
    grid-wide kernels)."""
    m, fixed = beam(4, 40, 4)
    bad = MLP(seed=11)
    bad.params = np.random.default_rng(0).normal(0.0, 30.0, NUM_PARAMS).astype(np.float32)
    runs = {}
    for learned in (False, True):
        s = mg.Solver(m, mg_params(levels=3, use_graph=graph))
        s.set_fixed(fixed)
        s.set_coarse_split(split)
        if learned:
            s.set_learned_smoother(bad, 0.5)
        for a, b in capsule_path(12, start=(0.0, 0.0, 1.3)):
            s.set_capsule(a, b, 0.3)
            s.step()
        runs[learned] = s.positions()
        if learned:
            v, fb = s.learned_stats()
            assert v == 12 * 10 and fb == v, (v, fb)
        s.close()
    assert np.array_equal(runs[True], runs[False])


@pytest.mark.parametrize("graph", [1, 0])
def test_guard_falls_back_to_plain_mixed(lib, graph):
    """Mixed precision: with a network that fails every check, every frame
    is the plain mixed-precision solver's frame, bit for bit."""
    m, fixed = beam(4, 40, 4)
    bad = MLP(seed=12)
    bad.params = np.random.default_rng(1).normal(0.0, 30.0, NUM_PARAMS).astype(np.float32)
    p = mg_params(levels=3, precision=mg.PRECISION_MIXED, refinement_passes=2, use_graph=graph)
    runs = {}
    for learned in (False, True):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        if learned:
            s.set_learned_smoother(bad, 0.5)
        for a, b in capsule_path(10, start=(0.0, 0.0, 1.3)):
            s.set_capsule(a, b, 0.3)
            s.step()
        runs[learned] = s.positions_f64()
        if learned:
            v, fb = s.learned_stats()
            assert v == 10 * 10 * 2 and fb == v, (v, fb)
        s.close()
    assert np.array_equal(runs[True], runs[False])


@pytest.mark.parametrize("precision", [mg.PRECISION_MIXED, mg.PRECISION_FP32])
@pytest.mark.parametrize("wild", [False, True])
def test_profiled_frame_equals_graph_frame(lib, trained, wild, precision):
    """A profiled frame (captured in two parts around the learned solve's
    decision, no conditional node) advances the run exactly as a frame of
    the solver's own graph, with and without the plain fallback; the
    profile lists the frame's kernels, the fallback's when it ran."""
    m, fixed = beam(4, 40, 4)
    net = trained[0]
    if wild:
        net = MLP(seed=13)
        net.params = np.random.default_rng(2).normal(0.0, 30.0, NUM_PARAMS).astype(np.float32)
    p = mg_params(levels=3, precision=precision, refinement_passes=1)
    path = capsule_path(6, start=(0.0, 0.0, 1.3))
    mixed = precision == mg.PRECISION_MIXED
    runs = []
    for profiled in (False, True):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_learned_smoother(net, 0.5)
        for f, (a, b) in enumerate(path):
            s.set_capsule(a, b, 0.3)
            if profiled and f == 4:
                failed_before = s.learned_stats()[1]
                prof = s.profile_frame()
                assert prof["k_ls_sweep_tc"][1] == 2 * p.iterations
                # the plain solve of the fallback runs exactly when a check of this frame failed
                plain_kernel = "k_mx_update" if mixed else "k_l0_sweep_rg"
                assert (plain_kernel in prof) == (s.learned_stats()[1] > failed_before)
                if wild:
                    assert plain_kernel in prof
            else:
                s.step()
        runs.append((s.positions_f64() if mixed else s.positions(), s.learned_stats()))
        s.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_learned_mixed_matches_oracle(lib, oracle_built, trained):
    """Learned smoother + mixed precision (FP64 residual, 3 refinement passes)
    against the FP64 oracle running plain V-cycles with the same passes: the
    global steps converge, so the smoother does not show in the frames."""
    net = trained[0]
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, precision=mg.PRECISION_MIXED, refinement_passes=3)
    s = mg.Solver(m, p)
    s.set_fixed(fixed)
    s.set_learned_smoother(net, 0.5)
    o = Oracle(m, p)
    o.set_fixed(fixed)
    path = capsule_path(60, start=(0.0, 0.0, 1.4))
    for f in range(60):
        for solver in (s, o):
            solver.set_capsule(*path[f], 0.3)
            solver.step()
    err = np.abs(s.positions_f64() - o.positions()).max()
    assert err < 1e-5 * m.bbox_diagonal(), err
    assert np.array_equal(np.nonzero(s.contact_flags())[0], np.nonzero(o.contact_flags())[0])
    v, fb = s.learned_stats()
    assert v == 60 * 10 * 3 and fb <= v // 10, (v, fb)
    s.close()


def test_time_kernel_learned_cycle_restores_state(lib, trained):
    """Replay timing of the learned cycle's kernels (tensor-core sweep, guard)
    leaves the frames and the guard's statistics as they were."""
    net = trained[0]
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, precision=mg.PRECISION_MIXED, refinement_passes=1)
    path = capsule_path(8, start=(0.0, 0.0, 1.4))
    runs = []
    for timed in (False, True):
        s = mg.Solver(m, p)
        s.set_fixed(fixed)
        s.set_learned_smoother(net, 0.5)
        for f, (a, b) in enumerate(path):
            s.set_capsule(a, b, 0.3)
            if timed and f == 4:
                for name in ("k_ls_sweep_tc", "k_ls_guard_residual<false>", "k_mx_residual", "k_coarse_vcycle"):
                    us, k = s.time_kernel(name, 8)
                    assert us > 0.0 and k >= 1, (name, us, k)
                assert s.time_kernel("k_ls_sweep_tc", 1)[1] == 2 * p.iterations
            s.step()
        runs.append((s.positions_f64(), s.learned_stats()))
        s.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_select_sweeps_on_the_gpu(lib, trained):
    """The sweep-count tuner with the real solver and its default timer: every
    candidate within the bar is timed, the choice is the fastest of them, and
    the choice's error is the one measured."""
    from multigridsoftbody_b200 import sweeps

    net = trained[0]
    m, fixed = beam(4, 40, 4)
    p = mg_params(levels=3, precision=mg.PRECISION_MIXED, refinement_passes=1)
    path = capsule_path(20, start=(0.0, 0.0, 1.3), seed=5)

    def tool(f):
        a, b = path[f % len(path)]
        return a[None], b[None], np.array([0.3], np.float32)

    out = sweeps.select_sweeps(m, fixed, p, net, tool, frames=10, bar=1e-3)
    for fam in ("learned_mixed", "plain_fp32"):
        rows = out[fam]["candidates"]
        timed = [r for r in rows if "ms_per_frame" in r]
        assert all(r["ms_per_frame"] > 0.0 for r in timed)
        assert all(("ms_per_frame" in r) == (r["err_over_diag"] <= 1e-3) for r in rows)
        if timed:
            assert out[fam]["chosen"] == min(timed, key=lambda r: r["ms_per_frame"])
    assert out["learned_mixed"]["chosen"] is not None
