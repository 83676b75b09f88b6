"""Bone-surface binding oracle (the reference's target_mode="mesh" driver,
mg/kernel.py:267-347) on the CPU: closest points are on their face and no
farther than a dense sample of the surface, the bind offset reconstructs the
query on the bind-time surface, and the target follows a rigid bone motion."""
from collections import Counter

import numpy as np
from scipy.spatial import cKDTree

from oracle import oracle as O
from rlmusclev2_b200.meshgen import capsule_surface


def _surface():
    v, t = capsule_surface([0.0, 0.0, 0.0], [0.3, 0.2, 1.0], 0.1, 0.02, n_around=12, n_lat=3)
    return v, t


def test_capsule_surface_is_closed_and_outward():
    v, t = _surface()
    edges = Counter()
    for a, b, c in t:
        for x, y in ((a, b), (b, c), (c, a)):
            edges[tuple(sorted((int(x), int(y))))] += 1
    assert set(edges.values()) == {2}
    n = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    assert (np.einsum("ij,ij->i", n, v[t].mean(1) - v.mean(0)) > 0).all()


def test_bind_closest_points_and_reconstruction():
    v, t = _surface()
    rng = np.random.default_rng(0)
    q = (rng.normal(size=(1500, 3)) * 0.06).astype(np.float32)
    face, uv, loc = O.bone_bind(q, v, t, 1.0)
    A, B, Cc = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    assert (uv >= 0).all() and (uv.sum(1) <= 1 + 1e-6).all()
    cp = uv[:, :1] * A[face] + uv[:, 1:] * B[face] + (1 - uv.sum(1, keepdims=True)) * Cc[face]
    s = rng.random((300, 2))
    m = s.sum(1) > 1
    s[m] = 1 - s[m]
    pts = (s[:, 0, None, None] * A[None] + s[:, 1, None, None] * B[None]
           + (1 - s.sum(1))[:, None, None] * Cc[None]).reshape(-1, 3)
    dd, _ = cKDTree(pts).query(q)
    assert (np.linalg.norm(q - cp, axis=1) <= dd + 1e-6).all()
    tgt, bf, _, _ = O.bone_slide_targets(q, face, uv, face, uv, loc, 0.005, 0, 1.0, v, t)
    assert np.abs(tgt - q).max() < 1e-6
    # nothing within max_dist: face 0 and zeros, as the reference writes
    far = np.array([[5.0, 5.0, 5.0]], np.float32)
    f2, uv2, l2 = O.bone_bind(far, v, t, 0.1)
    assert f2[0] == 0 and not uv2.any() and not l2.any()


def test_target_follows_a_rigid_bone_and_slides_within_range():
    v, t = _surface()
    rng = np.random.default_rng(1)
    q = (rng.normal(size=(800, 3)) * 0.05).astype(np.float32)
    face, uv, loc = O.bone_bind(q, v, t, 1.0)
    th = 0.4
    T = np.zeros((1, 3, 4))
    T[0, :, :3] = [[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]]
    T[0, :, 3] = [0.01, -0.02, 0.03]
    vb = O.bone_pose(v, np.zeros(v.shape[0], np.int32), T)
    tgt, _, _, _ = O.bone_slide_targets(q, face, uv, face, uv, loc, 0.005, 0, 1.0, vb, t)
    assert np.abs(tgt - (q @ T[0, :, :3].T + T[0, :, 3])).max() < 1e-6
    # reproject: a muscle point that drifted re-binds only within slide_range of its anchor
    moved = q + np.float32(0.002) * rng.normal(size=q.shape).astype(np.float32)
    _, bf, buv, loc2 = O.bone_slide_targets(moved, face, uv, face, uv, loc, 0.004, 1, 1.0, v, t)
    A, B, Cc = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    anc = uv[:, :1] * A[face] + uv[:, 1:] * B[face] + (1 - uv.sum(1, keepdims=True)) * Cc[face]
    new = buv[:, :1] * A[bf] + buv[:, 1:] * B[bf] + (1 - buv.sum(1, keepdims=True)) * Cc[bf]
    slid = (bf != face) | (np.abs(buv - uv).max(1) > 0)
    assert slid.any() and (~slid).any()
    assert (np.linalg.norm(new - anc, axis=1)[slid] <= 0.004 + 1e-6).all()
