"""Synthetic meshes standing in for the reference's (absent) muscle assets.

Seeded generators with the shapes, sizes and value distributions of the
benchmark configurations: a jittered box muscle, a humanV2-scale scene of
ellipsoidal muscles with a fascia shell and capsule bones.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Kuhn/Freudenthal split of a hex into 6 tets along the (0,0,0)-(1,1,1)
# diagonal; conforming between neighbouring hexes that use the same split.
_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def hex_to_tets(corner_index) -> np.ndarray:
    """corner_index(dx,dy,dz) -> array of vertex ids (one per hex).  Returns
    (6*nhex, 4) tets [a, b, c, d] with d the far corner."""
    out = []
    for p in _PERMS:
        step = [0, 0, 0]
        path = [corner_index(0, 0, 0)]
        for ax in p:
            step[ax] = 1
            path.append(corner_index(*step))
        out.append(np.stack(path, axis=1))
    return np.concatenate(out, axis=0)


def orient_tets(pos: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Swap pts[0], pts[1] where det[p0-p3, p1-p3, p2-p3] < 0 so every tet is
    positively oriented with the pt3 reference vertex."""
    t = tets.copy()
    p = pos[t].astype(np.float64)
    d = np.linalg.det(np.stack([p[:, 0] - p[:, 3], p[:, 1] - p[:, 3], p[:, 2] - p[:, 3]], axis=-1))
    neg = d < 0
    t[neg, 0], t[neg, 1] = tets[neg, 1], tets[neg, 0]
    return t


@dataclass
class BoxMuscle:
    verts: np.ndarray
    tets: np.ndarray
    fiber_per_tet: np.ndarray
    stopped: np.ndarray
    meta: dict = field(default_factory=dict)


def box_muscle(nx=8, ny=8, nz=32, spacing=0.0025, jitter=0.0002, seed=0, pin_frac=0.05) -> BoxMuscle:
    """Box muscle: (nx+1)(ny+1)(nz+1) grid verts at ``spacing`` (m), 6 tets per
    hex, rest positions jittered by U(-jitter, jitter) from ``seed``, fiber +z,
    vertices in the first/last ``pin_frac`` of the z extent stopped."""
    vid = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)  # noqa: E731
    i = np.arange((nx + 1) * (ny + 1) * (nz + 1))
    gi, gj, gk = i % (nx + 1), (i // (nx + 1)) % (ny + 1), i // ((nx + 1) * (ny + 1))
    verts = np.stack([gi, gj, gk], 1).astype(np.float64) * spacing
    rng = np.random.default_rng(seed)
    verts = (verts + rng.uniform(-jitter, jitter, size=verts.shape)).astype(np.float32)
    hi, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    tets = hex_to_tets(lambda dx, dy, dz: vid(hi + dx, hj + dy, hk + dz))
    tets = orient_tets(verts, tets).astype(np.int32)
    fiber = np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (tets.shape[0], 1))
    z = verts[:, 2]
    zr = (z - z.min()) / (z.max() - z.min())
    stopped = ((zr < pin_frac) | (zr > 1.0 - pin_frac)).astype(np.int32)
    return BoxMuscle(verts, tets, fiber, stopped, dict(nx=nx, ny=ny, nz=nz, spacing=spacing, seed=seed))
