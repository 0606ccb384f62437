"""Sweep counts picked by accuracy: the second half of the project's autotuner.

`Solver.autotune` picks the coarse-kernel shape of a given configuration by
timing; `select_sweeps` picks the configuration itself (Jacobi sweeps per
level and V-cycles per PD iteration) for each solver family, the learned
smoother with mixed precision and the plain FP32 multigrid, with the same
rule for both: run every candidate from rest over a tool path, compare the
positions with a converged solver (mixed precision, 6 FP64-residual V-cycles
per PD iteration, plain smoother), time the candidates whose max vertex error
(the largest Euclidean distance of a vertex from its converged position) stays
within `bar` x the bounding-box diagonal, and choose the fastest.

The reference has no counterpart: its solver runs fixed iteration counts
(`PDSolver.cpp:166`, 20 Jacobi iterations per frame).  Give the selection a
tool path other than the one a measurement then times.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .api import Solver

ERROR_BAR = 1e-5                                                         # x bbox diagonal
LEARNED_CANDIDATES = (((2, 2), 1), ((1, 1), 1), ((1, 1), 2), ((2, 2), 2))  # ((pre, post), passes)
PLAIN_CANDIDATES = (((2, 2), 1), ((2, 2), 2), ((1, 1), 1), ((1, 1), 2), ((1, 1), 3), ((2, 2), 3))


def max_vertex_error(x, ref) -> float:
    """The largest Euclidean distance between a vertex of x[V, 3] and the same vertex of ref[V, 3]."""
    d = np.asarray(x, np.float64) - np.asarray(ref, np.float64)
    return float(np.sqrt((d * d).sum(axis=1)).max()) if d.size else 0.0


def apply_tool(solver, poses) -> None:
    """poses = (a[k, 3], b[k, 3], r[k]): one capsule per body."""
    a, b, r = poses
    if len(r) == 1:
        solver.set_capsule(a[0], b[0], float(r[0]))
    else:
        solver.set_capsules(a, b, r)


def variant_params(base, sweeps, passes, learned):
    """A copy of `base` with (pre, post) sweeps, `passes` V-cycles per PD iteration and the precision of
    the family (mixed for the learned smoother, FP32 for the plain multigrid)."""
    p = type(base).from_buffer_copy(base)
    p.pre_sweeps, p.post_sweeps = sweeps
    p.refinement_passes = passes
    p.precision = _lib.PRECISION_MIXED if learned else _lib.PRECISION_FP32
    return p


def variant_key(sweeps, passes, learned) -> str:
    return "%s_%dpass_%d+%d" % ("learned_mixed" if learned else "plain_fp32", passes, sweeps[0], sweeps[1])


def run_positions(mesh, fixed, p, net, tool, frames, solver_cls=Solver):
    """Positions (FP64 array) after `frames` frames from rest, and the learned-smoother counters."""
    s = solver_cls(mesh, p)
    s.set_fixed(fixed)
    if net is not None:
        s.set_learned_smoother(net, 0.5)
    for f in range(frames):
        apply_tool(s, tool(f))
        s.step()
    x = s.positions_f64() if p.precision == _lib.PRECISION_MIXED else s.positions().astype(np.float64)
    stats = s.learned_stats() if net is not None else None
    s.close()
    return x, stats


def converged_positions(mesh, fixed, base, tool, frames, solver_cls=Solver):
    """The converged solver: mixed precision, 6 FP64-residual V-cycles (2+2 sweeps) per PD iteration."""
    return run_positions(mesh, fixed, variant_params(base, (2, 2), 6, True), None, tool, frames, solver_cls)[0]


def time_frames(mesh, fixed, p, net, tool, frames=60, warm=10, tune=True, solver_cls=Solver) -> float:
    """Default timer: ms per frame (the solver's own per-frame CUDA events) after an autotuned shape."""
    s = solver_cls(mesh, p)
    s.set_fixed(fixed)
    if net is not None:
        s.set_learned_smoother(net, 0.5)
    if tune:
        s.autotune(frames=5)
    for f in range(warm):
        apply_tool(s, tool(f))
        s.step()
    total = 0.0
    for k in range(frames):
        apply_tool(s, tool(warm + k))
        s.step()
        total += s.last_frame_ms()
    s.close()
    return total / frames


def select_sweeps(mesh, fixed, base, net, tool, time_fn=None, bar=ERROR_BAR, frames=100,
                  learned_candidates=LEARNED_CANDIDATES, plain_candidates=PLAIN_CANDIDATES, solver_cls=Solver,
                  time_all=False, margin=1.0):
    """For each family, every candidate's max vertex error / bbox diagonal after `frames` frames from
    rest against the converged solver -- the largest over the tool paths when `tool` is a list of tool
    callbacks --, the frame time (time_fn(params, net) in ms; default `time_frames` on the first path)
    of those within `bar` (of every candidate with `time_all`, so that the margins can be read), and the
    fastest candidate within margin x bar as the family's choice (None when none is within it): a
    margin below 1 keeps forms whose error sits just under the bar on these paths, and may exceed it
    on others, out of the choice.  `net` is the learned smoother (None skips that family)."""
    tools = list(tool) if isinstance(tool, (list, tuple)) else [tool]
    if time_fn is None:
        def time_fn(p, netx):
            return time_frames(mesh, fixed, p, netx, tools[0], solver_cls=solver_cls)
    refs = [converged_positions(mesh, fixed, base, t, frames, solver_cls) for t in tools]
    diag = mesh.bbox_diagonal()
    out = {"frames": frames, "bar": bar, "paths": len(tools), "margin": margin,
           "error": "max over vertices of the Euclidean distance / bbox diagonal, worst over the paths"}
    families = [("plain_fp32", plain_candidates, False)]
    if net is not None:
        families.insert(0, ("learned_mixed", learned_candidates, True))
    for fam, cands, learned in families:
        rows = []
        for sweeps, passes in cands:
            p = variant_params(base, sweeps, passes, learned)
            errs = []
            for t, ref in zip(tools, refs):
                x, _ = run_positions(mesh, fixed, p, net if learned else None, t, frames, solver_cls)
                errs.append(max_vertex_error(x, ref) / diag)
            err = max(errs)
            row = {"key": variant_key(sweeps, passes, learned), "sweeps": list(sweeps), "passes": passes,
                   "err_over_diag": err, "err_per_path": errs, "within_bar": bool(err <= bar)}
            if row["within_bar"] or time_all:
                row["ms_per_frame"] = float(time_fn(p, net if learned else None))
            rows.append(row)
        ok = [r for r in rows if r["err_over_diag"] <= margin * bar]
        out[fam] = {"candidates": rows, "chosen": min(ok, key=lambda r: r["ms_per_frame"]) if ok else None}
    return out
