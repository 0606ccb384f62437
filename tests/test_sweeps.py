"""The sweep-count selection (multigridsoftbody_b200.sweeps.select_sweeps) on a
fake solver class, no GPU: each family gets the fastest candidate whose error
against the converged solver stays within the bar, candidates outside the bar
are not timed, and a family with no candidate within the bar gets no choice."""
import ctypes

import pytest

import numpy as np

from multigridsoftbody_b200 import sweeps


class FakeParams(ctypes.Structure):
    _fields_ = [("pre_sweeps", ctypes.c_int32), ("post_sweeps", ctypes.c_int32),
                ("refinement_passes", ctypes.c_int32), ("precision", ctypes.c_int32)]


class FakeMesh:
    def bbox_diagonal(self):
        return 10.0


def fake_solver(error_of, axes=(1.0, 0.0, 0.0)):
    """A solver class that ends at positions error_of(params, learned) x axes away from the converged ones."""

    class Solver:
        def __init__(self, mesh, p):
            self.p = p
            self.learned = False

        def set_fixed(self, fixed):
            pass

        def set_learned_smoother(self, net, ratio):
            self.learned = True

        def set_capsule(self, a, b, r):
            self.scale = float(a[0]) if a[0] != 0 else 1.0   # a path can scale the error

        def step(self):
            pass

        def _x(self):
            converged = (self.p.refinement_passes == 6 and not self.learned)
            e = 0.0 if converged else error_of(self.p, self.learned) * getattr(self, "scale", 1.0)
            return np.tile(np.asarray(axes, np.float64) * e, (4, 1))

        def positions_f64(self):
            return self._x()

        def positions(self):
            return self._x().astype(np.float32)

        def learned_stats(self):
            return (1, 0)

        def close(self):
            pass

    return Solver


def tool(f):
    z = np.zeros((1, 3), np.float32)
    return z, z, np.array([0.3], np.float32)


def test_fastest_candidate_within_the_bar():
    def err(p, learned):   # error / diag = value / 10
        if learned:
            return 5e-5 if p.pre_sweeps == 1 else 4e-5              # both within 1e-5 * 10
        return 2e-4 / (p.refinement_passes * p.pre_sweeps)          # within the bar from 2 x 2+2 / 3 x ... on

    def cost(p, net):
        return p.refinement_passes * (p.pre_sweeps + 1.0) + (0.5 if net is not None else 0.0)

    timed = []

    def time_fn(p, net):
        timed.append((p.pre_sweeps, p.refinement_passes, net is not None))
        return cost(p, net)

    base = FakeParams(2, 2, 1, 1)
    out = sweeps.select_sweeps(FakeMesh(), None, base, object(), tool, time_fn, frames=2, solver_cls=fake_solver(err))
    assert out["learned_mixed"]["chosen"]["key"] == "learned_mixed_1pass_1+1"
    # plain: 2+2 x 1 pass has 1e-5 (bar met exactly: <=), 1+1 x 1 pass 2e-5 (not timed)
    assert out["plain_fp32"]["chosen"]["key"] == "plain_fp32_1pass_2+2"
    assert (1, 1, False) not in timed
    for fam in ("learned_mixed", "plain_fp32"):
        for r in out[fam]["candidates"]:
            assert ("ms_per_frame" in r) == (r["err_over_diag"] <= sweeps.ERROR_BAR) == r["within_bar"]


def test_no_candidate_within_the_bar():
    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), object(), tool, lambda p, net: 1.0,
                               frames=2, solver_cls=fake_solver(lambda p, learned: 1.0))
    assert out["learned_mixed"]["chosen"] is None and out["plain_fp32"]["chosen"] is None


def test_without_a_network_only_the_plain_family():
    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), None, tool, lambda p, net: 1.0,
                               frames=2, solver_cls=fake_solver(lambda p, learned: 0.0))
    assert "learned_mixed" not in out and out["plain_fp32"]["chosen"] is not None


def test_error_is_the_vertex_distance():
    """An error spread over all three axes counts with its Euclidean length: 0.8e-5 per axis is within a
    1e-5 bar coordinate by coordinate, but the vertex is 1.39e-5 away, so no candidate qualifies."""
    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), object(), tool, lambda p, net: 1.0,
                               frames=2, solver_cls=fake_solver(lambda p, learned: 0.8e-4, axes=(1.0, 1.0, 1.0)))
    for fam in ("learned_mixed", "plain_fp32"):
        assert out[fam]["chosen"] is None
        for r in out[fam]["candidates"]:
            assert abs(r["err_over_diag"] - 0.8e-5 * np.sqrt(3.0)) < 1e-12
    assert sweeps.max_vertex_error(np.array([[3.0, 4.0, 0.0], [0.0, 0.0, 1.0]]), np.zeros((2, 3))) == 5.0


def test_time_all_times_every_candidate():
    """With time_all every candidate carries its frame time; the choice still comes from within the bar."""
    def err(p, learned):
        return 0.0 if p.refinement_passes >= 2 else 1.0

    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), None, tool,
                               lambda p, net: 10.0 - p.refinement_passes, frames=2, solver_cls=fake_solver(err),
                               time_all=True)
    rows = out["plain_fp32"]["candidates"]
    assert all("ms_per_frame" in r for r in rows)
    assert out["plain_fp32"]["chosen"]["key"] == "plain_fp32_3pass_1+1"
    assert not any(r["within_bar"] for r in rows if r["passes"] == 1)


def test_worst_path_decides():
    """With several tool paths a candidate's error is its worst one: 0.6e-5 on one path and 1.2e-5 on
    another is outside a 1e-5 bar."""
    def path(scale):
        def tool(f):
            a = np.array([[scale, 0.0, 0.0]], np.float32)
            return a, a, np.array([0.3], np.float32)
        return tool

    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), None, [path(1.0), path(2.0)],
                               lambda p, net: 1.0, frames=2, solver_cls=fake_solver(lambda p, learned: 0.6e-4))
    for r in out["plain_fp32"]["candidates"]:
        assert r["err_per_path"] == pytest.approx([0.6e-5, 1.2e-5]) and not r["within_bar"]
    assert out["plain_fp32"]["chosen"] is None and out["paths"] == 2


def test_margin_keeps_forms_near_the_bar_out():
    """With margin 0.5 a form at 0.8 x bar is timed (within the bar) but not chosen; the slower form at
    0.4 x bar is."""
    def err(p, learned):   # error / diag = value / 10
        return 0.8e-4 if p.refinement_passes == 1 else 0.4e-4

    out = sweeps.select_sweeps(FakeMesh(), None, FakeParams(2, 2, 1, 1), None, tool,
                               lambda p, net: float(p.refinement_passes), frames=2, solver_cls=fake_solver(err),
                               margin=0.5)
    rows = {r["key"]: r for r in out["plain_fp32"]["candidates"]}
    assert rows["plain_fp32_1pass_2+2"]["within_bar"] and "ms_per_frame" in rows["plain_fp32_1pass_2+2"]
    assert out["plain_fp32"]["chosen"]["passes"] == 2 and out["margin"] == 0.5


def test_held_out_contraction_counts_and_ratios():
    """learned.held_out_contraction steps the solver along the path and summarises |r_after|/|r_before|
    over every learned V-cycle of every frame, with the solver's failed-check count."""
    from multigridsoftbody_b200.learned import held_out_contraction

    class FakeSolver:
        def __init__(self, mesh, params):
            self.frames = 0
            self.closed = False

        def set_fixed(self, mask):
            pass

        def set_learned_smoother(self, net, ratio):
            self.ratio = ratio

        def set_capsule(self, a, b, r):
            pass

        def step(self):
            self.frames += 1

        def learned_cycle_norms(self):   # two cycles per frame: ratios 0.1 and 0.6 (the second fails)
            return np.array([10.0, 1.0, 0.0]), np.array([1.0, 0.6, 0.0])

        def learned_stats(self):
            return 3 * self.frames, self.frames

        def close(self):
            self.closed = True

    path = [(np.zeros(3, np.float32), np.ones(3, np.float32))] * 5
    out = held_out_contraction(object(), None, None, None, path, solver_cls=FakeSolver)
    assert out["failed_checks"] == 5 and out["cycles"] == 15
    assert abs(out["ratio_max"] - 0.6) < 1e-12 and abs(out["ratio_p50"] - 0.35) < 1e-12
