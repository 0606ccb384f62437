"""Scene builders shared by the tests (configs of the workload at test sizes)."""
from __future__ import annotations

import numpy as np

import multigridsoftbody_b200 as mg


def beam(nx, ny, nz, half_len=10.0):
    m = mg.box_mesh(nx, ny, nz, (-1.0, -half_len, -1.0), (1.0, half_len, 1.0))
    fixed = (np.abs(m.positions[:, 1] - half_len) < 1e-5).astype(np.uint8)
    return m, fixed


def capsule_path(frames, start=(0.0, 0.0, 3.0), dz=-0.02, sigma=0.005, half_length=4.0, seed=1):
    """Capsule along x (segment length 2*half_length) moving -z with seeded jitter."""
    rng = np.random.default_rng(seed)
    c = np.array(start, np.float64)
    out = []
    for _ in range(frames):
        c = c + np.array([0.0, 0.0, dz]) + rng.normal(0.0, sigma, 3)
        a = (c - [half_length, 0, 0]).astype(np.float32)
        b = (c + [half_length, 0, 0]).astype(np.float32)
        out.append((a, b))
    return out


def mg_params(levels, iterations=10, gravity=(0.0, -9.8, 0.0), **kw):
    return mg.default_params(mg.SOLVER_MULTIGRID, levels=levels, iterations=iterations, gravity=gravity, **kw)
