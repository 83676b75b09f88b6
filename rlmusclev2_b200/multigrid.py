"""Two-level hpbd multigrid of MultiGridSim (mg/mg.py:744-1079) on the device.

Per substep, after the prediction: restrict the fine state onto the cage
(Galerkin least squares, snapshot q_j, kinematic pin of the coarse Dirichlet
nodes), ``mg_coarse_iters`` Jacobi ARAP-SVD sweeps of the cage (its own tile
engine, pins held by zero inverse mass; with mg_coarse_attach_beta != 0 each
sweep is followed by the soft attach of the referenced nodes), then add the
coarse displacement back onto the fine vertices (delta prolongation) and
re-pin.  The restricted
bone target that drives the coarse pins is recomputed once per frame (it is
constant across a frame's substeps).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as capi
from .builder import collect_raw_constraints
from .engine import XpbdSolver
from .meshgen import Cage, cage_for_config, coarse_in_fine_embedding


def _restrict_host(cage: Cage, x: np.ndarray, prior: np.ndarray) -> np.ndarray:
    """Host regularised Galerkin restriction (setup only):
    prior + Minv P^T (x - P prior)."""
    emb = cage.cage_idx >= 0
    t = cage.coarse_tet[cage.cage_idx[emb]]
    w = np.concatenate([(1.0 - cage.uvw[emb].astype(np.float64).sum(1))[:, None], cage.uvw[emb]], 1)
    prior = prior.astype(np.float64)
    r = x[emb].astype(np.float64) - sum(w[:, k:k + 1] * prior[t[:, k]] for k in range(4))
    b = np.zeros((cage.coarse_pos.shape[0], 3))
    for k in range(4):
        np.add.at(b, t[:, k], w[:, k:k + 1] * r)
    out = np.zeros_like(b)
    starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
    for s0 in starts:
        base, dim, off = cage.blk_base[s0], cage.blk_dim[s0], cage.blk_matoff[s0]
        M = cage.minv_flat[off:off + dim * dim].astype(np.float64).reshape(dim, dim)
        out[base:base + dim] = M @ b[base:base + dim]
    return prior + out


def node_mass_redistribute(pos, tet, total_mass) -> np.ndarray:
    """mg.py:56-68: node mass = 1/4 of incident |tet volume| (pt0 reference),
    scaled so the nodes carry total_mass."""
    r = pos[tet].astype(np.float64)
    Dm = np.stack([r[:, 1] - r[:, 0], r[:, 2] - r[:, 0], r[:, 3] - r[:, 0]], axis=-1)
    vol = np.abs(np.linalg.det(Dm)) / 6.0
    m = np.zeros(pos.shape[0])
    np.add.at(m, tet.reshape(-1), np.repeat(vol / 4.0, 4))
    tot = m.sum()
    if tot > 0:
        m *= total_mass / tot
    return m.astype(np.float32)


class DeviceMultigrid:
    def __init__(self, sim, spacing: float = 0.016):
        self.sim = sim
        cfg = sim.cfg
        # a baked cage file (coarse_npz_path) or the lattice cage; "pinv" blocks
        # are the reference's restriction as written, "tikhonov" the default
        cage = cage_for_config(sim.scene, {**cfg, "mg_cage_spacing": spacing},
                               operator=str(cfg.get("mg_restrict_operator", "tikhonov")))
        self.cage = cage
        ncoarse = cage.coarse_pos.shape[0]
        # FAS rest of the coarse ARAP = restriction of the fine rest (mg.py:813-829)
        q0 = _restrict_host(cage, sim.pos0_np, cage.coarse_pos).astype(np.float32)
        self.q0 = q0
        mass = node_mass_redistribute(cage.coarse_pos, cage.coarse_tet, sim.total_mass)
        # coarse Dirichlet pins restricted from the fine pins (mg.py:842-868)
        emb = cage.cage_idx >= 0
        corners = cage.coarse_tet[cage.cage_idx[emb]]
        w4 = np.abs(np.concatenate([(1.0 - cage.uvw[emb].astype(np.float64).sum(1))[:, None],
                                    cage.uvw[emb].astype(np.float64)], 1))
        wacc = np.zeros(ncoarse)
        np.add.at(wacc, corners.reshape(-1), w4.reshape(-1))
        fine_pin = sim.pin_active_np.astype(np.float64)[emb]
        pacc = np.zeros(ncoarse)
        np.add.at(pacc, corners.reshape(-1), (fine_pin[:, None] * w4).reshape(-1))
        with np.errstate(divide="ignore", invalid="ignore"):
            frac = np.where(wacc > 1e-9, pacc / wacc, 0.0)
        pin_frac = float(cfg.get("mg_coarse_pin_frac", 0.5))
        self.coarse_pin = ((frac >= pin_frac) & (wacc > 1e-9)).astype(np.int32)
        # coarse Neumann attach (mg.py:216, 1047-1062): after every coarse sweep the
        # nodes with a nonzero restriction column move by beta x (target - pos)
        # toward their restricted bone target; 0 = pure ARAP relax
        self.beta = float(cfg.get("mg_coarse_attach_beta", 0.0))
        self.attach_nodes = np.nonzero(wacc > 1e-9)[0]
        table = collect_raw_constraints(q0, cage.coarse_tet, [dict(type="tetarapsvd", name="arap",
                                                                    stiffness=sim.mu)]).sorted_by_type()
        # the cage's per-tet corrections stay far below its extent (its cells are
        # 16 mm, a smooth correction of the fine state), so its accumulator is
        # sized by the extent alone: a quantum of 1.5e-8 m on the 535k-tet scenes,
        # where 128 cage edges (3.5 m) would give 6e-8 m.  Coarse corrections
        # below half a quantum are lost (a dead zone), and the multigrid scene's
        # stiff tendon tets are sensitive to that at 6e-8 m.
        self.coarse = XpbdSolver(q0, cage.coarse_tet, table, mass=mass, dt=sim.dt, stopped=self.coarse_pin,
                                 device=sim.device, stream=sim._stream, acc_range=float(np.abs(q0).max()))
        self.iters = int(sim.mg_coarse_iters)
        # "hpbd": the cage is its own ARAP sim, delta-prolonged; "projection": the
        # fine state is reset to the prolonged restricted bone target each substep
        self.mode = str(getattr(sim, "mg_mode", "hpbd"))
        # step 1 of the V-cycle (mg.py:224-246, 1006-1012): "direct" restricts the
        # fine state (Galerkin least squares, or with mg_sync_restrict "c2f" the
        # coarse-in-fine barycentric readout), "galerkin" copies in the restricted
        # bone target, "none" leaves the coarse on its own state
        self.restrict_mode = str(cfg.get("mg_restrict_mode", "direct")).lower()
        if self.restrict_mode not in ("direct", "galerkin", "none"):
            raise ValueError(f"mg_restrict_mode must be 'direct', 'galerkin' or 'none', got {self.restrict_mode!r}")
        self.sync_restrict = str(cfg.get("mg_sync_restrict", "galerkin")).lower()
        if self.sync_restrict not in ("galerkin", "c2f"):
            raise ValueError(f"mg_sync_restrict must be 'galerkin' or 'c2f', got {self.sync_restrict!r}")
        self._build_device()

    def _build_device(self):
        sim, cage, co = self.sim, self.cage, self.coarse
        dev = sim.device
        ncoarse = cage.coarse_pos.shape[0]
        fl = sim.layout
        cl = co.layout
        emb = np.nonzero(cage.cage_idx >= 0)[0]
        t = cage.coarse_tet[cage.cage_idx[emb]]
        w = np.concatenate([(1.0 - cage.uvw[emb].astype(np.float64).sum(1))[:, None],
                            cage.uvw[emb].astype(np.float64)], 1).astype(np.float32)
        # restriction CSR per coarse vertex (cage order), fine ids in fine library order
        rows = t.reshape(-1)
        fine = np.repeat(fl.inv[emb], 4)
        ww = w.reshape(-1)
        order = np.lexsort((fine, rows))
        r_ptr = np.zeros(ncoarse + 1, np.int64)
        r_ptr[1:] = np.cumsum(np.bincount(rows, minlength=ncoarse))
        # prolongation per fine vertex (fine library order)
        p_idx = np.full((sim.n_verts, 4), -1, np.int32)
        p_w = np.zeros((sim.n_verts, 4), np.float32)
        p_idx[fl.inv[emb]] = cl.inv[t]
        p_w[fl.inv[emb]] = w
        starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
        blk_ptr = np.r_[cage.blk_base[starts], ncoarse].astype(np.int32)
        blk_moff = cage.blk_matoff[starts].astype(np.int32)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self._t = dict(r_ptr=T(r_ptr.astype(np.int32)), r_fine=T(fine[order].astype(np.int32)),
                       r_w=T(ww[order].astype(np.float32)), blk_ptr=T(blk_ptr), blk_moff=T(blk_moff),
                       minv=T(cage.minv_flat), coarse_lib=T(cl.inv.astype(np.int32)), p_idx=T(p_idx), p_w=T(p_w))
        self._t["resid"] = torch.zeros((sim.n_verts, 4), dtype=torch.float32, device=dev)
        self._t["rhs"] = torch.zeros((ncoarse, 4), dtype=torch.float32, device=dev)
        g = capi.XpbdCage()
        g.n_fine, g.n_coarse, g.n_blocks = sim.n_verts, ncoarse, int(blk_moff.shape[0])
        g.max_block = int(np.diff(blk_ptr).max())
        for k in ("r_ptr", "r_fine", "r_w", "blk_ptr", "blk_moff", "minv", "coarse_lib", "p_idx", "p_w", "resid", "rhs"):
            setattr(g, k, self._t[k].data_ptr())
        self.g = g
        self.prev = torch.zeros((ncoarse, 4), dtype=torch.float32, device=dev)
        pin4 = np.zeros((ncoarse, 4), np.float32)
        pin4[:, :3] = self.q0  # prior of the first target restriction
        pin4[:, 3] = self.coarse_pin
        self.pin4 = T(pin4[cl.perm])
        self.attach_idx = T(cl.inv[self.attach_nodes].astype(np.int32))
        self.g_c2f = None
        if self.sync_restrict == "c2f":
            # the coarse vertices embedded in fine rest tets (mg.py:897-898, 903-938):
            # the absolute prolongation with the roles swapped reads them off the fine mesh
            ct, cw = coarse_in_fine_embedding(sim.pos0_np, sim.tet_np, cage.coarse_pos)
            c_idx = np.empty((ncoarse, 4), np.int32)
            c_w = np.empty((ncoarse, 4), np.float32)
            c_idx[cl.inv] = fl.inv[ct]
            c_w[cl.inv] = cw
            self._t["c2f_idx"], self._t["c2f_w"] = T(c_idx), T(c_w)
            g2 = capi.XpbdCage.from_buffer_copy(g)
            g2.n_fine = ncoarse
            g2.p_idx, g2.p_w = self._t["c2f_idx"].data_ptr(), self._t["c2f_w"].data_ptr()
            self.g_c2f = g2

    def refresh_target(self):
        """Coarse Dirichlet targets = restriction of the fine bone targets (mg.py:1028-1045)."""
        s = self.sim
        capi.check(s._lib.xpbd_mg_restrict(C.byref(self.g), C.c_void_p(s._pin_tgt.data_ptr()),
                                           C.c_void_p(self.pin4.data_ptr()), None, None, s._sp))

    def vcycle(self, pin_fine: bool):
        """Restrict + coarse solve + delta prolong (+ fine re-pin); with
        mg_mode="projection" (mg.py:1263-1320) the restricted bone target,
        prolonged absolute onto the embedded fine vertices (+ fine re-pin)."""
        s, co = self.sim, self.coarse
        vf = s._vflags.data_ptr() if (pin_fine and s._vflags is not None) else None
        pt = s._pin_tgt.data_ptr() if (pin_fine and s._pin_tgt is not None) else None
        if self.mode == "projection":
            capi.check(s._lib.xpbd_mg_prolong_delta(C.byref(self.g), C.c_void_p(self.pin4.data_ptr()), None,
                                                    C.c_void_p(s._pos4.data_ptr()), C.c_void_p(vf) if vf else None,
                                                    C.c_void_p(pt) if pt else None, s._sp))
            return
        if self.restrict_mode == "direct" and self.g_c2f is None:
            capi.check(s._lib.xpbd_mg_restrict(C.byref(self.g), C.c_void_p(s._pos4.data_ptr()),
                                               C.c_void_p(co._pos4.data_ptr()), C.c_void_p(self.prev.data_ptr()),
                                               C.c_void_p(self.pin4.data_ptr()), s._sp))
        else:
            src = None
            if self.restrict_mode == "direct":  # restrict_c2f_kernel (mg/kernel.py:43-60)
                capi.check(s._lib.xpbd_mg_prolong_delta(C.byref(self.g_c2f), C.c_void_p(s._pos4.data_ptr()), None,
                                                        C.c_void_p(co._pos4.data_ptr()), None, None, s._sp))
            elif self.restrict_mode == "galerkin":  # the restricted bone target (mg.py:1265-1295)
                src = C.c_void_p(self.pin4.data_ptr())
            capi.check(s._lib.xpbd_mg_coarse_reset(C.byref(self.g), src, C.c_void_p(co._pos4.data_ptr()),
                                                   C.c_void_p(self.prev.data_ptr()),
                                                   C.c_void_p(self.pin4.data_ptr()), s._sp))
        if self.beta != 0.0:
            for _ in range(self.iters):  # ARAP sweep, then the soft attach (mg.py:1057-1062)
                co._fused_iterations(1)
                capi.check(s._lib.xpbd_blend_to_target(int(self.attach_idx.shape[0]),
                                                       C.c_void_p(self.attach_idx.data_ptr()), co.n_verts,
                                                       C.c_void_p(co._pos4.data_ptr()),
                                                       C.c_void_p(self.pin4.data_ptr()), C.c_float(self.beta),
                                                       s._sp))
        else:
            co._fused_iterations(self.iters)
        capi.check(s._lib.xpbd_mg_prolong_delta(C.byref(self.g), C.c_void_p(co._pos4.data_ptr()),
                                                C.c_void_p(self.prev.data_ptr()), C.c_void_p(s._pos4.data_ptr()),
                                                C.c_void_p(vf) if vf else None, C.c_void_p(pt) if pt else None,
                                                s._sp))
