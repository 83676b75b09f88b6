"""Fascia shell sub-solver, ride mode (the reference's Fascia with
fascia_mode="ride", fascia/fascia.py:179-572): a Stable Neo-Hookean shell
whose vertices near the muscle are bound barycentrically to the closest
muscle-surface triangle (plus the signed normal gap) and follow it every
substep; the muscle is never pushed.  The shell runs on its own tile engine
(one more XpbdSolver on the parent's stream)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as capi
from .builder import collect_raw_constraints, lumped_mass


class FasciaRide:
    def __init__(self, parent, verts: np.ndarray, tets: np.ndarray, *, snh_mu: float, snh_lam: float,
                 snh_damp: float, total_mass: float, iterations: int, bind_max_dist: float):
        from .engine import XpbdSolver
        self.parent = parent
        self.iterations = int(iterations)
        verts = np.asarray(verts, np.float32)
        tets = np.asarray(tets, np.int32)
        table = collect_raw_constraints(verts, tets, [dict(type="snh", name="snh", mu=snh_mu, lam=snh_lam,
                                                           dampingratio=snh_damp)]).sorted_by_type()
        _, vols = lumped_mass(verts, tets, 1.0)
        density = float(total_mass) / float(max(vols.astype(np.float64).sum(), 1e-30))
        mass, _ = lumped_mass(verts, tets, density)
        # quasi-static shell (Fascia.integrate snapshots pprev only): no prediction, no velocity
        self.solver = XpbdSolver(verts, tets, table, mass=mass, dt=parent.dt, quasi_static=True,
                                 device=parent.device, stream=parent._stream)
        s = self.solver
        lib = parent._lib
        # muscle surface in the parent's library vertex order, bound at the muscle rest pose
        tris = parent.layout.inv[np.asarray(parent.scene.surface_tris, np.int64)].astype(np.int32)
        dev = parent.device
        self._stris = torch.from_numpy(np.ascontiguousarray(tris)).to(dev)
        q4 = np.zeros((s.n_verts, 4), np.float32)
        q4[:, :3] = verts[s.layout.perm]  # fascia library order
        q4d = torch.from_numpy(q4).to(dev)
        n = s.n_verts
        face = torch.zeros(n, dtype=torch.int32, device=dev)
        uv = torch.zeros((n, 2), dtype=torch.float32, device=dev)
        gap = torch.zeros(n, dtype=torch.float32, device=dev)
        ok = torch.zeros(n, dtype=torch.int32, device=dev)
        capi.check(lib.xpbd_surface_bind(n, C.c_void_p(q4d.data_ptr()), parent.NV,
                                         C.c_void_p(parent._rest4.data_ptr()), int(tris.shape[0]),
                                         C.c_void_p(self._stris.data_ptr()), C.c_float(bind_max_dist),
                                         C.c_void_p(face.data_ptr()), C.c_void_p(uv.data_ptr()),
                                         C.c_void_p(gap.data_ptr()), C.c_void_p(ok.data_ptr()), parent._sp))
        parent._stream.synchronize()
        bound = torch.nonzero(ok == 1).flatten().to(torch.int32)
        self.n_bound = int(bound.numel())
        self._bound = bound.contiguous()
        self._face = face[bound.long()].contiguous()
        self._uv = uv[bound.long()].contiguous()
        self._gap = gap[bound.long()].contiguous()

    def ride(self) -> None:
        """Snap the bound shell vertices onto the current muscle surface (_ride)."""
        if not self.n_bound:
            return
        p = self.parent
        capi.check(p._lib.xpbd_surface_ride(self.n_bound, C.c_void_p(self._bound.data_ptr()),
                                            C.c_void_p(self._face.data_ptr()), C.c_void_p(self._uv.data_ptr()),
                                            C.c_void_p(self._gap.data_ptr()), C.c_void_p(p._pos4.data_ptr()),
                                            C.c_void_p(self._stris.data_ptr()),
                                            C.c_void_p(self.solver._pos4.data_ptr()), p._sp))

    def substep(self) -> None:
        """build_program_ride (fascia.py:499-522): ride, snapshot pprev, then
        ``iterations`` x (SNH Jacobi iteration, ride)."""
        s = self.solver
        self.ride()
        with torch.cuda.stream(s._stream):
            s._prev4.copy_(s._pos4)
        for _ in range(self.iterations):
            s._fused_iteration()
            self.ride()

    def positions_np(self) -> np.ndarray:
        return self.solver.positions_np()
