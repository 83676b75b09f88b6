"""Fascia shell sub-solvers (the reference's Fascia, fascia/fascia.py:179-572).

Ride mode (FasciaRide): a Stable Neo-Hookean shell whose vertices near the
muscle are bound barycentrically to the closest muscle-surface triangle (plus
the signed normal gap) and follow it every substep; the muscle is never
pushed.  Squeeze mode (FasciaSqueeze): a shrunk ARAP + volume shell carried by
the bones that pulls the muscle surface with one-way glue.  Each shell runs on
its own tile engine (one more XpbdSolver on the parent's stream)."""
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

    def advect(self) -> None:
        """Per-frame bone advection: none in ride mode (fascia.py:528-529)."""

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


class FasciaSqueeze:
    """Fascia shell sub-solver, squeeze mode (the reference's legacy
    fascia_mode, fascia/fascia.py:311-441, 524-566): an ARAP-SVD + volume shell
    whose ARAP rest is shrunk by ``rest_scale``, carried by the skeleton (each
    shell vertex follows the bone target of its nearest muscle vertex, once per
    frame), held by a sparse set of bone anchors, and pulling the muscle
    surface toward it with one-way glue springs (only the muscle moves)."""

    def __init__(self, parent, verts: np.ndarray, tets: np.ndarray, *, rest_scale: float, arap_k: float,
                 arap_damp: float, vol_k: float, vol_damp: float, glue_k: float, total_mass: float,
                 iterations: int, anchor_count: int, rigid: np.ndarray | None = None):
        from scipy.spatial import cKDTree

        from .engine import XpbdSolver
        if not rest_scale > 0.0:
            raise ValueError(f"fascia_arap.rest_scale must be > 0, got {rest_scale}")
        self.parent = parent
        self.iterations = int(iterations)
        verts = np.asarray(verts, np.float32)
        tets = np.asarray(tets, np.int32)
        table = collect_raw_constraints(verts, tets, [
            dict(type="tetarapsvd", name="fascia_arap", stiffness=arap_k, dampingratio=arap_damp),
            dict(type="volume", name="fascia_volume", stiffness=vol_k, dampingratio=vol_damp)]).sorted_by_type()
        _, vols = lumped_mass(verts, tets, 1.0)
        density = float(total_mass) / float(max(vols.astype(np.float64).sum(), 1e-30))
        mass, _ = lumped_mass(verts, tets, density)
        self.solver = XpbdSolver(verts, tets, table, mass=mass, dt=parent.dt, quasi_static=True,
                                 device=parent.device, stream=parent._stream)
        s = self.solver
        if abs(rest_scale - 1.0) >= 1e-9:  # _apply_rest_shrink: B <- B / scale (ARAP rest only)
            with torch.cuda.stream(s._stream):
                for t in (s._t_b0, s._t_b1, s._t_b2):
                    t.mul_(1.0 / rest_scale)
        dev = parent.device
        pl, fl = parent.layout, s.layout
        mrest = parent.pos0_np
        # glue (_pair_surface): every muscle surface vertex to its nearest shell vertex, at the rest gap
        surf = np.unique(np.asarray(parent.scene.surface_tris, np.int64))
        gd, gf = cKDTree(verts).query(mrest[surf], k=1)
        self.n_glue = int(surf.size)
        self._gf = torch.from_numpy(fl.inv[gf].astype(np.int32)).to(dev)
        self._gm = torch.from_numpy(pl.inv[surf].astype(np.int32)).to(dev)
        self._grest = torch.from_numpy(gd.astype(np.float32)).to(dev)
        self._gcomp = torch.full((self.n_glue,), 1.0 / max(float(glue_k), 1e-30), dtype=torch.float32, device=dev)
        # bone follow: nearest muscle vertex (restricted to the pinned-target points when the
        # targets are cons frames, as the reference maps unpinned ones to the nearest pinned)
        cand = getattr(parent, "_cons_pts", None)
        cand = np.arange(parent.NV) if cand is None else np.asarray(cand, np.int64)
        _, loc = cKDTree(mrest[cand]).query(verts, k=1)
        follow_user = cand[loc]
        follow_lib = np.empty(s.n_verts, np.int64)  # per shell vertex in the shell's library order
        follow_lib[fl.inv] = pl.inv[follow_user]
        self._follow = torch.from_numpy(follow_lib.astype(np.int32)).to(dev)
        tgt = parent._pin_tgt
        if tgt is None:
            raise ValueError("fascia squeeze needs the muscle's per-vertex targets (a pin or belly attach)")
        with torch.cuda.stream(s._stream):
            self._prev = tgt[self._follow.long()].clone()
            self._prev[:, 3] = 0.0
        # bone anchors: the "rigid" group or a uniform subsample of count vertices
        rid = (np.asarray(rigid, np.int64) if rigid is not None else
               np.arange(0, verts.shape[0], max(1, verts.shape[0] // max(1, int(anchor_count))), dtype=np.int64))
        self.n_anchor = int(rid.size)
        self._alocal = torch.from_numpy(fl.inv[rid].astype(np.int32)).to(dev)
        self._acons = torch.from_numpy(pl.inv[follow_user[rid]].astype(np.int32)).to(dev)
        with torch.cuda.stream(s._stream):
            off = s._pos4[self._alocal.long()] - tgt[self._acons.long()]
            off[:, 3] = 0.0
            self._aoff = off.contiguous()
        s._stream.synchronize()

    def _p(self, t):
        return C.c_void_p(t.data_ptr())

    def advect(self) -> None:
        """advect_bone (fascia.py:524-533): once per frame, after the targets."""
        p, s = self.parent, self.solver
        capi.check(p._lib.xpbd_fascia_advect(s.n_verts, self._p(self._follow), self._p(p._pin_tgt), self._p(self._prev),
                                             self._p(s._pos4), p._sp))

    def substep(self) -> None:
        """build_program (fascia.py:535-566): anchors, snapshot pprev, then
        ``iterations`` x (ARAP + volume Jacobi iteration, one-way glue)."""
        p, s = self.parent, self.solver
        if self.n_anchor:
            capi.check(p._lib.xpbd_fascia_anchor(self.n_anchor, self._p(self._alocal), self._p(self._acons),
                                                 self._p(self._aoff), self._p(p._pin_tgt), self._p(s._pos4), p._sp))
        with torch.cuda.stream(s._stream):
            s._prev4.copy_(s._pos4)
        for _ in range(self.iterations):
            s._fused_iteration()
            capi.check(p._lib.xpbd_fascia_glue(self.n_glue, self._p(self._gf), self._p(self._gm), self._p(self._grest),
                                               self._p(self._gcomp), self._p(s._pos4), self._p(p._pos4),
                                               C.c_float(p.dt), C.c_float(p.omega), p._sp))

    def positions_np(self) -> np.ndarray:
        return self.solver.positions_np()
