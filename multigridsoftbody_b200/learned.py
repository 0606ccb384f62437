"""The learned smoother's network (mgsb_mlp_* in the C ABI): a per-vertex MLP
9 -> 64 -> 64 -> 3 with GELU, BF16 weights on the tensor cores, trained on
the GPU by the library's own forward/backward kernels and Adam."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

NUM_PARAMS = 4995


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = L.load()
        h = C.c_void_p()
        st = self._lib.mgsb_mlp_create(device, seed, C.byref(h))
        if st != 0:
            raise RuntimeError(f"mgsb_mlp_create failed: {L.STATUS.get(st, st)}")
        self.h = h

    def _check(self, st):
        if st != 0:
            msg = self._lib.mgsb_mlp_last_error(self.h)
            raise RuntimeError(f"{L.STATUS.get(st, st)}: {msg.decode() if msg else ''}")

    def close(self):
        if self.h:
            self._lib.mgsb_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.empty(NUM_PARAMS, np.float32)
        self._check(self._lib.mgsb_mlp_get_params(self.h, _fp(out), NUM_PARAMS))
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._lib.mgsb_mlp_set_params(self.h, _fp(p), p.shape[0]))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        y = np.empty((x.shape[0], 3), np.float32)
        self._check(self._lib.mgsb_mlp_forward(self.h, _fp(x), x.shape[0], _fp(y)))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, 3)
        g = np.empty(NUM_PARAMS, np.float32)
        loss = np.empty(1, np.float32)
        self._check(self._lib.mgsb_mlp_loss_grad(self.h, _fp(x), _fp(t), x.shape[0], _fp(g), _fp(loss)))
        return float(loss[0]), g

    def train(self, x, t, steps: int = 20000, batch: int = 4096, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 9)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, 3)
        losses = np.empty(steps, np.float32)
        self._check(self._lib.mgsb_mlp_train(self.h, _fp(x), _fp(t), x.shape[0], steps, batch, lr, seed, _fp(losses)))
        return losses


# ---------------------------------------------------------------------------
# The learned-smoother scene (organ-like blob) and the training pipeline
# ---------------------------------------------------------------------------
def blob_scene(levels: int = 5, precision: int = L.PRECISION_FP32, refinement_passes: int = 1, **overrides):
    """Blob from a 64x32x48 voxel grid (spacing 0.25) inside (x/6)^2+(y/3)^2+(z/4)^2 < 1 + 0.15 s(x,y,z)
    (seed-3 value noise, period 2), 6 tets per voxel; fixed x < -5; E 3e4, nu 0.45; gravity -9.8 along z;
    dt 1/60; multigrid with `levels` levels.  Returns (mesh, fixed mask, params)."""
    from .api import blob_mesh, default_params
    m = blob_mesh()
    fixed = (m.positions[:, 0] < -5.0).astype(np.uint8)
    p = default_params(L.SOLVER_MULTIGRID, levels=levels, gravity=(0.0, 0.0, -9.8), youngs_modulus=3e4,
                       poisson_ratio=0.45, precision=precision, refinement_passes=refinement_passes, **overrides)
    return m, fixed, p


def blob_tool_path(frames: int, seed: int, start=(0.0, 0.0, 3.3), dz: float = -0.02, sigma: float = 0.005,
                   half_length: float = 4.0):
    """Capsule r 0.3 along x (segment length 8) above the blob, moving -z 0.02 per frame plus
    N(0, sigma^2) jitter per axis (seeded)."""
    rng = np.random.default_rng(seed)
    c = np.array(start, np.float64)
    out = []
    for _ in range(frames):
        c = c + np.array([0.0, 0.0, dz]) + rng.normal(0.0, sigma, 3)
        out.append(((c - [half_length, 0, 0]).astype(np.float32), (c + [half_length, 0, 0]).astype(np.float32)))
    return out


def generate_pairs(runs: int = 32, frames: int = 40, every: int = 20, sweeps: int = 4, device: int = 0,
                   first_seed: int = 100):
    """Residual/correction pairs from the plain FP32 multigrid solver on `runs` seeded blob runs:
    every `every` frames, the pairs of the state after the frame (mgsb_smoother_pairs)."""
    from .api import Solver
    m, fixed, p = blob_scene()
    p.device = device
    xs, ts = [], []
    for r in range(runs):
        s = Solver(m, p)
        s.set_fixed(fixed)
        path = blob_tool_path(frames, seed=first_seed + r)
        for f in range(frames):
            s.set_capsule(*path[f], 0.3)
            s.step()
            if (f + 1) % every == 0:
                x, t = s.smoother_pairs(sweeps)
                xs.append(x)
                ts.append(t)
        s.close()
    return np.concatenate(xs), np.concatenate(ts)


def train_smoother(x, t, steps: int = 20000, batch: int = 4096, lr: float = 2e-3, seed: int = 0, device: int = 0):
    net = MLP(device=device, seed=seed)
    losses = net.train(x, t, steps=steps, batch=batch, lr=lr, seed=seed + 1)
    return net, losses


def held_out_contraction(net, mesh, fixed, params, tool_path, guard_ratio: float = 0.5, solver_cls=None):
    """How well `net` smooths inside the learned V-cycle on a held-out run: steps a solver with
    `params` (a learned form: mixed precision, its sweeps and passes) along `tool_path` ((a, b)
    capsule ends per frame, radius 0.3) and collects, per learned V-cycle, |r_after| / |r_before|
    (mgsb_learned_cycle_norms).  Returns {"failed_checks", "cycles", "ratio_p50", "ratio_p99",
    "ratio_max"}; fewer failed checks, then a lower 99th percentile, is better."""
    if solver_cls is None:
        from .api import Solver as solver_cls
    s = solver_cls(mesh, params)
    try:
        s.set_fixed(fixed)
        s.set_learned_smoother(net, guard_ratio)
        ratios = []
        for a, b in tool_path:
            s.set_capsule(a, b, 0.3)
            s.step()
            before, after = s.learned_cycle_norms()
            ok = before > 0
            ratios.extend((after[ok] / before[ok]).tolist())
        checks, failed = s.learned_stats()
    finally:
        s.close()
    r = np.asarray(ratios) if ratios else np.zeros(1)
    return {"failed_checks": int(failed), "cycles": int(checks), "ratio_p50": float(np.percentile(r, 50)),
            "ratio_p99": float(np.percentile(r, 99)), "ratio_max": float(r.max())}
