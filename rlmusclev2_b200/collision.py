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
