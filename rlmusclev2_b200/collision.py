"""Bone push-out through a grid signed-distance field.

Replaces the reference's AnimatedBoneMeshCollider (example/humanV2.py:319-418),
which refits a wp.Mesh of the bones every frame and queries
mesh_query_point_sign_normal per vertex (collision/sdf/kernel.py:122-170).
Here the bones are capsules whose union SDF is baked every frame into a
``res``^3 FP32 grid on the device (brick-culled, narrow band); the push-out
runs inside the fused per-vertex kernel: err = phi - contact_offset, and a
vertex with err < 0 (and depth <= max_push when max_push > 0) moves by
-err along the normalised trilinear gradient.  Vertices with inverse mass 0
are skipped, as in the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as capi


class GridSdfCollider:
    """Per-frame capsule-bone SDF on a cubic grid plus the push-out hook."""

    graph_safe = True  # bake + push are device launches only (the fused frame may capture them)

    def __init__(self, sim, centers, axes, halves, radii, *, res: int = 256, contact_offset: float = 0.0,
                 max_push: float = -1.0, band_cells: float = 3.0, margin: float = 0.02, bbox=None):
        self.sim = sim
        self.device = sim.device
        self.n_caps = len(radii)
        caps = (capi.XpbdCapsule * max(1, self.n_caps))()
        for i in range(self.n_caps):
            caps[i].center[:] = [float(x) for x in centers[i]]
            caps[i].axis[:] = [float(x) for x in axes[i]]
            caps[i].half = float(halves[i])
            caps[i].radius = float(radii[i])
        raw = bytes(caps)
        self._caps = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device)
        if bbox is None:
            lo, hi = sim.pos0_np.min(0), sim.pos0_np.max(0)
        else:
            lo, hi = np.asarray(bbox[0]), np.asarray(bbox[1])
        lo = lo - margin
        hi = hi + margin
        ext = float((hi - lo).max())
        self.res = int(res)
        self.h = ext / (self.res - 1)
        self.origin = lo.astype(np.float64)
        self.band = float(band_cells) * self.h
        self.phi = torch.empty((self.res, self.res, self.res), dtype=torch.float32, device=self.device)
        s = capi.XpbdSdf()
        s.phi = self.phi.data_ptr()
        s.nx = s.ny = s.nz = self.res
        s.origin[:] = [float(x) for x in self.origin]
        s.h = float(self.h)
        s.contact_offset = float(contact_offset)
        s.max_push = float(max_push)
        self._s = s
        self.transforms = None  # device (n_caps, 12) or None = rest pose

    def struct(self) -> capi.XpbdSdf:
        return self._s

    def bake(self) -> None:
        lib = self.sim._lib
        tr = None if self.transforms is None else C.c_void_p(self.transforms.data_ptr())
        capi.check(lib.xpbd_sdf_bake_capsules(C.byref(self._s), self.n_caps, C.c_void_p(self._caps.data_ptr()), tr,
                                              C.c_float(self.band), self.sim._sp))

    def __call__(self) -> None:
        """Push-out hook (collision_solvers entry, mg/mg.py:1366-1371)."""
        self.sim._vstep_sdf_only(self)


class BatchedSdfCollider:
    """One capsule-bone SDF grid per instance of a batch (its two bones), all
    baked in one launch; push-out reads each vertex's own grid."""

    graph_safe = True

    def __init__(self, sim, scene, *, contact_offset: float = 0.0, max_push: float = -1.0, band_cells: float = 3.0):
        self.sim = sim
        self.device = sim.device
        n = scene.n_inst
        self.caps_per_inst = 2
        caps = (capi.XpbdCapsule * (2 * n))()
        for i in range(2 * n):
            caps[i].center[:] = [float(x) for x in scene.bone_center[i]]
            caps[i].axis[:] = [float(x) for x in scene.bone_axis[i]]
            caps[i].half = float(scene.bone_half[i])
            caps[i].radius = float(scene.bone_radius[i])
        self._caps = torch.frombuffer(bytearray(bytes(caps)), dtype=torch.uint8).to(self.device)
        self.res = int(scene.sdf_res)
        self.frame = torch.from_numpy(np.ascontiguousarray(scene.sdf_frame, np.float32)).to(self.device)
        self.band = float(band_cells) * float(scene.sdf_frame[:, 3].max())
        self.phi = torch.empty((n, self.res, self.res, self.res), dtype=torch.float32, device=self.device)
        L = sim.layout
        self.vert_inst = torch.from_numpy(np.ascontiguousarray(scene.vert_inst[L.perm], np.int32)).to(self.device)
        s = capi.XpbdSdfBatch()
        s.phi, s.frame, s.vert_inst = self.phi.data_ptr(), self.frame.data_ptr(), self.vert_inst.data_ptr()
        s.n_inst, s.nx, s.ny, s.nz = n, self.res, self.res, self.res
        s.contact_offset, s.max_push = float(contact_offset), float(max_push)
        self._s = s
        self.transforms = None  # device (2 n_inst, 12) or None = rest pose

    def struct(self) -> capi.XpbdSdfBatch:
        return self._s

    def bake(self) -> None:
        tr = None if self.transforms is None else C.c_void_p(self.transforms.data_ptr())
        capi.check(self.sim._lib.xpbd_sdf_bake_capsules_batched(C.byref(self._s), self.caps_per_inst,
                                                                C.c_void_p(self._caps.data_ptr()), tr,
                                                                C.c_float(self.band), self.sim._sp))

    def __call__(self) -> None:
        """Push-out hook (collision_solvers entry)."""
        self.sim._sdf = self
        self.sim._vstep(capi.OP_SDF)


# ----------------------------------------------------------------------------
# Triangle-triangle DCD (UdcfDcdCollider, collision/udcf/solver.py:38-457)

from dataclasses import dataclass  # noqa: E402


@dataclass
class UdcfParams:
    """UdcfParams (udcf/solver.py:38-120); the BVH broadphase is the only one
    (use_bvh=True), the serial Gauss-Seidel variant is not on this path."""
    multiplier: float = 1.01
    friction_static: float = 0.5
    friction_dynamic: float = 0.4
    offset: float = 1.0e-6
    thickness: float = 0.0
    max_pairs: int = 1 << 20
    max_contacts: int = 1 << 18
    allow_self: bool = False
    jacobi_avg: bool = True
    gauss_seidel: bool = False
    max_push: float = 0.0
    use_bvh: bool = True
    # Library-specific: rebuild the LBVH (Morton sort + hierarchy) every n-th
    # broadphase and refit the boxes in between.  1 = the reference's
    # per-broadphase rebuild; the pair set is the same for any n.
    bvh_rebuild_every: int = 1


class DcdBuffers:
    """Device buffers and the XpbdDcd descriptor for ``n_tris`` triangles over
    a [n_verts][4] position buffer (library vertex ids)."""

    def __init__(self, lib, device, tris_lib: np.ndarray, n_verts: int, params: UdcfParams, box_lo, box_hi,
                 tri_group: np.ndarray | None = None):
        self.lib = lib
        self.p = params
        n = int(tris_lib.shape[0])
        sz = capi.XpbdDcdWorkspaceSizes()
        capi.check(lib.xpbd_dcd_workspace_query(n, C.byref(sz)))
        dev = device
        i32 = torch.int32
        self.t = dict(
            tris=torch.from_numpy(np.ascontiguousarray(tris_lib, np.int32)).to(dev),
            group=None if tri_group is None else torch.from_numpy(np.ascontiguousarray(tri_group, np.int32)).to(dev),
            pairs=torch.zeros((params.max_pairs, 2), dtype=i32, device=dev),
            counters=torch.zeros(8, dtype=i32, device=dev),  # n_pairs, n_contacts, status, total
            c_ids=torch.zeros((params.max_contacts, 8), dtype=i32, device=dev),
            c_data=torch.zeros((params.max_contacts, 12), dtype=torch.float32, device=dev),
            x_prev=torch.zeros((n_verts, 4), dtype=torch.float32, device=dev),
            dP=torch.zeros((n_verts, 4), dtype=torch.float32, device=dev),
            nodes=torch.zeros(int(sz.nodes_floats), dtype=torch.float32, device=dev),
            keys=torch.zeros(int(sz.keys), dtype=i32, device=dev), vals=torch.zeros(int(sz.keys), dtype=i32, device=dev),
            keys2=torch.zeros(int(sz.keys), dtype=i32, device=dev), vals2=torch.zeros(int(sz.keys), dtype=i32, device=dev),
            hist=torch.zeros(int(sz.hist), dtype=i32, device=dev),
            bbox=torch.zeros(int(sz.bbox_floats), dtype=torch.float32, device=dev),
            count=torch.zeros(int(sz.count), dtype=i32, device=dev),
            slots=torch.zeros(int(sz.slots), dtype=i32, device=dev),
            split=torch.zeros(int(sz.split), dtype=i32, device=dev))
        t = self.t
        d = capi.XpbdDcd()
        d.n_tris, d.n_verts, d.max_pairs, d.max_contacts = n, int(n_verts), params.max_pairs, params.max_contacts
        d.tris = t["tris"].data_ptr()
        d.tri_group = None if t["group"] is None else t["group"].data_ptr()
        d.allow_self, d.jacobi_avg = int(params.allow_self), int(params.jacobi_avg)
        d.thickness, d.offset_eps, d.multiplier = params.thickness, params.offset, params.multiplier
        d.friction_static, d.friction_dynamic, d.max_push = params.friction_static, params.friction_dynamic, params.max_push
        d.box_lo[:] = [float(x) for x in box_lo]
        d.box_hi[:] = [float(x) for x in box_hi]
        cp = t["counters"].data_ptr()
        d.pairs, d.n_pairs, d.n_contacts, d.status = t["pairs"].data_ptr(), cp, cp + 4, cp + 8
        d.ws_total = cp + 12
        d.c_ids, d.c_data, d.x_prev, d.dP = (t["c_ids"].data_ptr(), t["c_data"].data_ptr(), t["x_prev"].data_ptr(),
                                             t["dP"].data_ptr())
        d.ws_nodes, d.ws_keys, d.ws_vals = t["nodes"].data_ptr(), t["keys"].data_ptr(), t["vals"].data_ptr()
        d.ws_keys2, d.ws_vals2, d.ws_hist = t["keys2"].data_ptr(), t["vals2"].data_ptr(), t["hist"].data_ptr()
        d.ws_bbox = t["bbox"].data_ptr()
        d.ws_count, d.ws_slots = t["count"].data_ptr(), t["slots"].data_ptr()
        d.ws_split = t["split"].data_ptr()
        self._built = False
        self.d = d

    def broadphase(self, pos4: torch.Tensor, snapshot_prev: bool, stream, refit_only: bool = False) -> None:
        """Boxes, LBVH and pair list; ``refit_only`` keeps the last rebuild's
        Morton order and hierarchy (the first call always rebuilds)."""
        self.d.refit_only = int(bool(refit_only) and self._built)
        capi.check(self.lib.xpbd_dcd_broadphase(C.byref(self.d), C.c_void_p(pos4.data_ptr()), int(snapshot_prev),
                                                stream))
        self._built = True

    def broadphase_launches(self, snapshot_prev: bool = True, refit_only: bool = False) -> int:
        """Kernels one xpbd_dcd_broadphase call launches: snapshot copy, boxes,
        cooperative sort (not when refitting), leaf permute, build or refit,
        counting traversal, the count scan (2 launches, 3 above 4096
        triangles), fill pass, total."""
        n = int(self.d.n_tris)
        scan = 2 + (1 if n > 4096 else 0)
        sort = 0 if refit_only else 1
        return int(snapshot_prev) + 2 + sort + (1 if n > 1 else 0) + 1 + scan + 2

    def narrow_respond(self, pos4: torch.Tensor, stream) -> None:
        capi.check(self.lib.xpbd_dcd_narrow_respond(C.byref(self.d), C.c_void_p(pos4.data_ptr()), stream))

    def reset(self) -> None:
        """Zero the counters (pair and contact counts, status word) and the
        sort's grid-barrier words, on the current stream: after a barrier
        timeout the next broadphase then runs with full barriers."""
        self.t["counters"].zero_()
        self.t["hist"].zero_()

    def counters(self) -> dict:
        c = self.t["counters"].cpu().numpy()
        return {"n_pairs": int(c[0]), "n_contacts": int(c[1]), "status": int(c[2])}


class UdcfDcdCollider:
    """Self-collision DCD of a sim's surface triangles (movable vs movable with
    allow_self, the configuration of the synthetic humanV2 scene).  Register
    ``solve`` in ``sim.collision_solvers_iter``: it rebuilds the LBVH on the
    first fine iteration of each substep and resolves contacts every
    iteration (udcf/solver.py:365-440)."""

    def __init__(self, sim, surface_tris: np.ndarray, params: UdcfParams | None = None, margin: float = 0.05):
        self.params = params or UdcfParams(allow_self=True)
        if self.params.gauss_seidel:
            raise NotImplementedError("the serial Gauss-Seidel DCD variant is not on the sm_100a path")
        if not self.params.allow_self:
            raise ValueError("UdcfDcdCollider: no static body and allow_self=False -> nothing to collide")
        self.sim = sim
        tris = np.asarray(surface_tris, np.int64).reshape(-1, 3)
        self.n_tris = tris.shape[0]
        lo = sim.pos0_np.min(0) - margin
        hi = sim.pos0_np.max(0) + margin
        self.buf = DcdBuffers(sim._lib, sim.device, sim.layout.inv[tris], sim.n_verts, self.params, lo, hi)
        self._peak = 0
        self._n_broad = 0  # broadphase calls so far (rebuild cadence; a captured frame repeats its pattern)

    def solve(self, i_iter: int = 0) -> None:
        s = self.sim
        if i_iter == 0:
            every = max(1, int(self.params.bvh_rebuild_every))
            self.buf.broadphase(s._pos4, True, s._sp, refit_only=(self._n_broad % every) != 0)
            self._n_broad += 1
        self.buf.narrow_respond(s._pos4, s._sp)

    __call__ = solve

    def stats(self) -> dict:
        """udcf/solver.py:442-457: counts of the last pass (one device sync)."""
        self.sim.synchronize()
        c = self.buf.counters()
        p = self.params
        if c["status"] & capi.STATUS_BARRIER_TIMEOUT:
            with torch.cuda.stream(self.sim._stream):
                self.buf.reset()
            self.sim._stream.synchronize()
            raise RuntimeError("[udcf_dcd] the broadphase sort gave up waiting at a grid barrier; "
                               "pairs were invalid (the counters and barrier words have been cleared)")
        if c["status"] & capi.STATUS_STACK_OVERFLOW:
            print("[udcf_dcd] WARNING: BVH traversal stack overflow")
        if c["n_pairs"] > p.max_pairs or c["n_contacts"] > p.max_contacts:
            print(f"[udcf_dcd] WARNING: overflow pairs={c['n_pairs']}/{p.max_pairs} "
                  f"contacts={c['n_contacts']}/{p.max_contacts} -- raise UdcfParams caps")
        return {"n_pairs": min(c["n_pairs"], p.max_pairs), "n_contacts": min(c["n_contacts"], p.max_contacts),
                "status": c["status"]}
