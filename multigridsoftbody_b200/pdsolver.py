"""Mirror of the reference's solver interface (MultiGridSoftBody/src/PDSolver.h:70-110,
Collider.h:5-36) on top of the C ABI, so code written against the reference's
PDSolver reads the same: construct, set the public m_* fields, Init(...),
then Step() per frame and read m_tetVertPos / m_tetVertIsCollide.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .api import Solver, TetMesh, default_params


class SphereCollider:
    """SphereCollider (Collider.h:5-20): a moving sphere tool."""

    def __init__(self, pos, radius: float):
        self.m_position = np.asarray(pos, np.float32).copy()
        self.m_position_last = self.m_position.copy()
        self.m_radius = float(radius)
        self.m_active = True

    def MoveDelta(self, delta) -> None:  # Collider.cpp:9-17
        self.m_position_last = self.m_position.copy()
        self.m_position = self.m_position + np.asarray(delta, np.float32)

    def MoveTo(self, target) -> None:  # Collider.cpp:19-27
        self.m_position_last = self.m_position.copy()
        self.m_position = np.asarray(target, np.float32).copy()


class SphereFixer(SphereCollider):
    """SphereFixer (Collider.h:32-36): vertices inside are fixed; not a collider."""

    def __init__(self, pos, radius: float):
        super().__init__(pos, radius)
        self.m_active = False


class PDSolver:
    """Jacobi/Chebyshev PD solver with the reference's constants and API.

    Fields default to PDSolver::Init's constants (PDSolver.cpp:166-176) and may
    be changed before Init(), as in the reference.
    """

    def __init__(self):
        p = default_params(L.SOLVER_REFERENCE_JACOBI)
        self.m_iterNum = p.iterations
        self.m_dt = p.dt
        self.m_damping = p.damping
        self.m_volumnStiffness = p.volume_stiffness
        self.m_collisionStiffness = p.collision_stiffness
        self.m_rho = p.cheb_rho
        self.m_gravityX, self.m_gravityY, self.m_gravityZ = (float(g) for g in p.gravity)
        self.m_sphereFixers: list[SphereFixer] = []
        self.m_sphereColliders: list[SphereCollider] = []
        self._solver: Solver | None = None

    # PDSolver::Init (PDSolver.cpp:164-200)
    def Init(self, tetVertPos, tetIdx, tetFaceIdx=None, tetFaceOppositeTetVertIdx=None) -> None:
        pos = np.asarray(tetVertPos, np.float32).reshape(-1, 3)
        tets = np.asarray(tetIdx, np.int32).reshape(-1, 4)
        self.m_tetVertNum = pos.shape[0]
        self.m_tetNum = tets.shape[0]
        self.m_tetIndex = tets.reshape(-1).copy()
        self.m_outsideTriIndex = None if tetFaceIdx is None else np.asarray(tetFaceIdx, np.int32).reshape(-1)
        self.m_outsideTriOppositeVertId = (None if tetFaceOppositeTetVertIdx is None
                                           else np.asarray(tetFaceOppositeTetVertIdx, np.int32).reshape(-1))
        p = default_params(L.SOLVER_REFERENCE_JACOBI, iterations=int(self.m_iterNum), dt=float(self.m_dt),
                           damping=float(self.m_damping), volume_stiffness=float(self.m_volumnStiffness),
                           collision_stiffness=float(self.m_collisionStiffness), cheb_rho=float(self.m_rho),
                           gravity=(self.m_gravityX, self.m_gravityY, self.m_gravityZ))
        self._solver = Solver(TetMesh(pos, tets), p)
        pre = self._solver.precompute()
        self.m_tetInvD3x3 = pre["inv"].reshape(-1)
        self.m_tetInvD3x4 = pre["ac"].reshape(-1)
        self.m_tetVolume = pre["volume"]
        self.m_tetVertMass = pre["mass"]
        self.m_tetVolumeDiag = pre["diag"]
        self.m_tetVertPos = pos.reshape(-1).copy()
        self.SetFixedVert()

    # PDSolver::SetFixedVert (PDSolver.cpp:134-162): inside any fixer sphere -> fixed
    def SetFixedVert(self) -> None:
        pos = self.m_tetVertPos.reshape(-1, 3).astype(np.float32)
        fixed = np.zeros(pos.shape[0], np.uint8)
        for sp in self.m_sphereFixers:
            d = np.sqrt(((pos - sp.m_position[None, :]) ** 2).sum(1))
            fixed |= (d < sp.m_radius).astype(np.uint8)
        self.m_tetVertFixed = np.where(fixed > 0, 0.0, 1.0).astype(np.float32)  # reference flag: 0 = fixed
        self._solver.set_fixed(fixed)

    def _sync_params(self) -> None:
        """The reference reads its public fields at every Step, so assignments after Init take effect on
        the next frame; here a changed field goes to the solver through mgsb_set_params."""
        p = self._solver.get_params()
        want = {"iterations": int(self.m_iterNum), "dt": float(self.m_dt), "damping": float(self.m_damping),
                "volume_stiffness": float(self.m_volumnStiffness),
                "collision_stiffness": float(self.m_collisionStiffness), "cheb_rho": float(self.m_rho)}
        g = (float(self.m_gravityX), float(self.m_gravityY), float(self.m_gravityZ))
        changed = {k: v for k, v in want.items() if getattr(p, k) != type(v)(np.float32(v) if isinstance(v, float) else v)}
        if tuple(float(x) for x in p.gravity) != tuple(float(np.float32(x)) for x in g):
            changed["gravity"] = g
        if changed:
            self._solver.set_params(**changed)

    # PDSolver::Step (PDSolver.cpp:243-293) incl. the render readback
    def Step(self) -> None:
        self._sync_params()
        cols = [c for c in self.m_sphereColliders]
        if cols:
            self._solver.set_spheres(np.stack([c.m_position for c in cols]), [c.m_radius for c in cols],
                                     [1 if c.m_active else 0 for c in cols])
        else:
            self._solver.set_spheres(np.zeros((0, 3), np.float32), np.zeros(0, np.float32))
        self._solver.step()
        self.RenderOnce()

    # runCpyTetVertForRender (PDSolver.cu:261-268)
    def RenderOnce(self) -> None:
        pos, flags = self._solver.frame()   # positions and contact flags in one readback
        self.m_tetVertPos = pos.reshape(-1)
        self.m_tetVertIsCollide = flags
        self.m_tetVertCollisionDepth = self._solver.collision_depth()

    @property
    def solver(self) -> Solver:
        return self._solver
