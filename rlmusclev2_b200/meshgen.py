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


def fix_tet_winding(vertices: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """The reference loader's winding rule (util/mesh_utils.py:16-32): swap
    pts[0] and pts[1] where (p1-p0) x (p2-p0) . (p3-p0) < 0.  Meshes loaded
    by the reference pass through it, so their pt3-referenced rest volumes
    det[p0-p3, p1-p3, p2-p3]/6 come out negative."""
    t = np.array(tets, copy=True)
    p0, p1, p2, p3 = (vertices[t[:, k]] for k in range(4))
    bad = np.einsum("ij,ij->i", np.cross(p1 - p0, p2 - p0), p3 - p0) < 0.0
    t[bad, 0], t[bad, 1] = tets[bad, 1], tets[bad, 0]
    return t


def ramp_activation(mask: np.ndarray, frame: int, start: int, end: int) -> np.ndarray:
    """RampActivationSource.per_tet (util/activation.py:28-44):
    clamp((frame - start) / max(1, end - start), 0, 1) * mask."""
    a = min(1.0, max(0.0, (int(frame) - int(start)) / max(1, int(end) - int(start))))
    return (a * np.asarray(mask, np.float32)).astype(np.float32)


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


# --------------------------------------------------------------------------
# humanV2-scale scene: ellipsoidal muscles + fascia shell + capsule bones


def _seg_dist(p0, p1, q0, q1) -> float:
    """Distance between segments p0p1 and q0q1 (clamped closest points)."""
    d1, d2, r = p1 - p0, q1 - q0, p0 - q0
    a, e, f = d1 @ d1, d2 @ d2, d2 @ r
    c, b = d1 @ r, d1 @ d2
    den = a * e - b * b
    s = np.clip((b * f - c * e) / den, 0.0, 1.0) if den > 1e-18 else 0.0
    t = (b * s + f) / e if e > 1e-18 else 0.0
    if t < 0.0:
        t, s = 0.0, np.clip(-c / a, 0.0, 1.0) if a > 1e-18 else 0.0
    elif t > 1.0:
        t, s = 1.0, np.clip((b - c) / a, 0.0, 1.0) if a > 1e-18 else 0.0
    return float(np.linalg.norm((p0 + d1 * s) - (q0 + d2 * t)))


def _rand_rot(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def axis_angle(axis: np.ndarray, ang: float) -> np.ndarray:
    a = axis / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * (K @ K)


def clipped_ellipsoid_lattice(L: float, r1: float, r2: float, h: float):
    """Hex lattice over the ellipsoid's box, cells with centre inside kept,
    6 tets per cell.  Returns local verts (x along the long axis) and tets."""
    nx = max(2, int(np.ceil(L / h)))
    ny = max(2, int(np.ceil(2 * r1 / h)))
    nz = max(2, int(np.ceil(2 * r2 / h)))
    hx, hy, hz = L / nx, 2 * r1 / ny, 2 * r2 / nz
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    cx = -L / 2 + (ci + 0.5) * hx
    cy = -r1 + (cj + 0.5) * hy
    cz = -r2 + (ck + 0.5) * hz
    keep = (cx / (L / 2)) ** 2 + (cy / r1) ** 2 + (cz / r2) ** 2 <= 1.0
    ci, cj, ck = ci[keep], cj[keep], ck[keep]
    gid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    tets = hex_to_tets(lambda dx, dy, dz: gid(ci + dx, cj + dy, ck + dz))
    used, tets = np.unique(tets, return_inverse=True)
    tets = tets.reshape(-1, 4)
    gi = used // ((ny + 1) * (nz + 1))
    gj = (used // (nz + 1)) % (ny + 1)
    gk = used % (nz + 1)
    verts = np.stack([-L / 2 + gi * hx, -r1 + gj * hy, -r2 + gk * hz], 1)
    return verts, tets


def boundary_faces(tets: np.ndarray) -> np.ndarray:
    """Faces used by exactly one tet, wound outward (right-hand normal points
    away from the tet's fourth vertex)."""
    f = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    opp = np.concatenate([tets[:, 3], tets[:, 2], tets[:, 1], tets[:, 0]])
    key = np.sort(f, axis=1)
    _, idx, cnt = np.unique(key, axis=0, return_index=True, return_counts=True)
    sel = idx[cnt == 1]
    return f[sel], opp[sel]


def orient_faces_outward(pos: np.ndarray, faces: np.ndarray, opp: np.ndarray) -> np.ndarray:
    a, b, c = pos[faces[:, 0]], pos[faces[:, 1]], pos[faces[:, 2]]
    n = np.cross(b - a, c - a)
    inward = np.einsum("ij,ij->i", n, pos[opp] - a) > 0
    out = faces.copy()
    out[inward, 1], out[inward, 2] = faces[inward, 2], faces[inward, 1]
    return out


def extrude_shell(pos: np.ndarray, faces: np.ndarray, thickness: float, min_quality: float = 0.25):
    """Prism shell outward of a closed surface: new inner and outer vertex
    layers, 3 tets per prism with the vertex-id diagonal rule (conforming).
    Prisms whose worst tet has a quality V / l_max^3 below ``min_quality`` x
    the shell's median (slivers at the staircase folds of a lattice surface,
    where the averaged vertex normal lies almost in a face's plane) are left
    out.  Returns the shell vertices, its tets and, per shell vertex, the
    surface vertex it comes from."""
    sv, inv = np.unique(faces, return_inverse=True)
    tri = inv.reshape(-1, 3)
    p = pos[sv]
    a, b, c = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
    fn = np.cross(b - a, c - a)
    vn = np.zeros_like(p)
    for k in range(3):
        np.add.at(vn, tri[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    n = p.shape[0]
    verts = np.concatenate([p, p + thickness * vn])
    t = np.sort(tri, axis=1)
    a0, b0, c0 = t[:, 0], t[:, 1], t[:, 2]
    a1, b1, c1 = a0 + n, b0 + n, c0 + n
    tets = np.concatenate([np.stack([a0, b0, c0, c1], 1), np.stack([a0, b0, b1, c1], 1),
                           np.stack([a0, a1, b1, c1], 1)])
    x = verts.astype(np.float64)
    e = [x[tets[:, j]] - x[tets[:, i]] for i, j in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(e[0], e[1]), e[2])) / 6.0
    q = vol / np.max([np.linalg.norm(v, axis=1) for v in e], axis=0) ** 3
    nf = tri.shape[0]
    qp = q.reshape(3, nf).min(0)
    keep = np.tile(qp >= min_quality * np.median(q), 3)
    used, tets = np.unique(tets[keep], return_inverse=True)
    return verts[used], tets.reshape(-1, 4), np.concatenate([sv, sv])[used]


@dataclass
class Scene:
    verts: np.ndarray            # (NV,3) float32, metres
    tets: np.ndarray             # (NT,4) int32, positively oriented (pt3 reference)
    tet_part: np.ndarray         # (NT,) muscle index, or -1 for fascia tets
    vert_part: np.ndarray        # (NV,) muscle index, or -1 for fascia verts
    v_tendon: np.ndarray         # (NV,) 1 on tendon verts (end 5% of a muscle's axis)
    v_fiber: np.ndarray          # (NV,3) unit fiber direction
    surface_tris: np.ndarray     # (NTRI,3) outward muscle surface triangles
    bone_center: np.ndarray      # (NB,3)
    bone_axis: np.ndarray        # (NB,3) unit
    bone_half: np.ndarray        # (NB,) half segment length
    bone_radius: np.ndarray      # (NB,)
    vert_bone: np.ndarray        # (NV,2) bones at the two ends of the vertex's muscle
    vert_bw: np.ndarray          # (NV,) blend weight of vert_bone[:,1] (axial coordinate 0..1)
    traj: dict                   # bone trajectory parameters
    aniso_muscle: int
    meta: dict = field(default_factory=dict)
    muscle_rot: np.ndarray | None = None     # (M,3,3) local->world rotation (column 0 = long axis)
    muscle_center: np.ndarray | None = None  # (M,3)
    muscle_len: np.ndarray | None = None     # (M,)
    act_sched: np.ndarray | None = None      # optional knots (every 8 frames from frame 1) of the fiber activation

    @property
    def n_bones(self) -> int:
        return int(self.bone_center.shape[0])

    def bone_surface(self, n_around: int = 16, n_lat: int = 4):
        """Rest triangle surfaces of all capsule bones, for the bone-surface
        binding (target_mode="mesh"): (verts [NBV,3], tris [NBT,3], vert_bone
        [NBV])."""
        vs, ts, vb, off = [], [], [], 0
        for b in range(self.n_bones):
            v, t = capsule_surface(self.bone_center[b], self.bone_axis[b], float(self.bone_half[b]),
                                   float(self.bone_radius[b]), n_around, n_lat)
            vs.append(v)
            ts.append(t + off)
            vb.append(np.full(v.shape[0], b, np.int32))
            off += v.shape[0]
        return np.concatenate(vs), np.concatenate(ts).astype(np.int32), np.concatenate(vb)

    def bone_transforms(self, frame: float) -> np.ndarray:
        """(NB,3,4) rigid transforms [R | t] at ``frame``: x -> R (x - c) + c + d,
        the identity at the start frame (targets bind to the rest pose there)."""
        tr = self.traj
        f = float(frame) - float(tr.get("start_frame", 1))
        ang = tr["rot_amp"] * (np.sin(tr["rot_w"] * f + tr["rot_phase"]) - np.sin(tr["rot_phase"]))
        a = tr["rot_axis"] / np.linalg.norm(tr["rot_axis"], axis=1, keepdims=True)
        K = np.zeros((a.shape[0], 3, 3))
        K[:, 0, 1], K[:, 0, 2], K[:, 1, 2] = -a[:, 2], a[:, 1], -a[:, 0]
        K[:, 1, 0], K[:, 2, 0], K[:, 2, 1] = a[:, 2], -a[:, 1], a[:, 0]
        R = np.eye(3) + np.sin(ang)[:, None, None] * K + (1.0 - np.cos(ang))[:, None, None] * (K @ K)
        d = (tr["tr_amp"] * (np.sin(tr["tr_w"] * f + tr["tr_phase"]) - np.sin(tr["tr_phase"])))[:, None] * tr["tr_dir"]
        c = np.asarray(self.bone_center, np.float64)
        out = np.zeros((self.n_bones, 3, 4))
        out[:, :, :3] = R
        out[:, :, 3] = c + d - np.einsum("bij,bj->bi", R, c)
        return out

    def targets(self, frame: float) -> np.ndarray:
        """Bone-driven target of every vertex at ``frame`` (float32, the device's
        operation order): (1-w) (R_a x + t_a) + w (R_b x + t_b)."""
        T = self.bone_transforms(frame).astype(np.float32)
        x = self.verts.astype(np.float32)
        out = []
        for k in range(2):
            Tb = T[self.vert_bone[:, k]]
            out.append(np.stack([((Tb[:, r, 0] * x[:, 0] + Tb[:, r, 1] * x[:, 1]) + Tb[:, r, 2] * x[:, 2]) + Tb[:, r, 3]
                                 for r in range(3)], 1))
        w = self.vert_bw.astype(np.float32)[:, None]
        return (out[0] + w * (out[1] - out[0])).astype(np.float32)

    def activation(self, frame: int, start: int = 1, end: int = 50) -> np.ndarray:
        """RampActivationSource (util/activation.py:28-44) on the aniso muscle's
        tets, or the piecewise-linear schedule act_sched when one is set."""
        if self.act_sched is not None:
            return (self.muscle_activation(frame)[self.aniso_muscle] * (self.tet_part == self.aniso_muscle)).astype(
                np.float32)
        return ramp_activation(self.tet_part == self.aniso_muscle, frame, start, end)

    def muscle_activation(self, frame: int, start: int = 1, end: int = 50) -> np.ndarray:
        """(n_muscles,) activation of every muscle (only the aniso muscle has a
        fiber constraint; the others are 0)."""
        out = np.zeros(self.muscle_rot.shape[0], np.float32)
        if self.act_sched is not None:
            f = (float(frame) - 1.0) / 8.0
            k = int(np.clip(np.floor(f), 0, self.act_sched.shape[0] - 2))
            u = float(np.clip(f - k, 0.0, 1.0))
            out[self.aniso_muscle] = (1.0 - u) * self.act_sched[k] + u * self.act_sched[k + 1]
        else:
            out[self.aniso_muscle] = min(1.0, max(0.0, (int(frame) - start) / max(1, end - start)))
        return out


def capsule_surface(c, axis, half: float, r: float, n_around: int = 16, n_lat: int = 4):
    """Closed triangle surface of a capsule (segment c +- half * axis, radius
    r): two hemispheres of n_lat latitude rings each joined by the cylinder,
    n_around vertices per ring plus the two poles.  Returns (verts, tris)."""
    c = np.asarray(c, np.float64)
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    e1 = np.cross(a, [1.0, 0.0, 0.0] if abs(a[0]) < 0.9 else [0.0, 1.0, 0.0])
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(a, e1)
    th = 2.0 * np.pi * np.arange(n_around) / n_around
    rad = np.cos(th)[:, None] * e1 + np.sin(th)[:, None] * e2
    rings = []
    for k in range(1, n_lat + 1):  # bottom hemisphere, pole side first, ends at the equator
        ph = -0.5 * np.pi + 0.5 * np.pi * k / n_lat
        rings.append(c - half * a + r * (np.sin(ph) * a + np.cos(ph) * rad))
    for k in range(n_lat):  # top hemisphere from its equator
        ph = 0.5 * np.pi * k / n_lat
        rings.append(c + half * a + r * (np.sin(ph) * a + np.cos(ph) * rad))
    verts = [c - (half + r) * a[None]] + rings + [c + (half + r) * a[None]]
    verts = np.concatenate(verts).astype(np.float32)
    top = verts.shape[0] - 1
    tris = []
    for j in range(n_around):  # bottom fan (outward normals)
        tris.append([0, 1 + (j + 1) % n_around, 1 + j])
    for q in range(len(rings) - 1):
        b0, b1 = 1 + q * n_around, 1 + (q + 1) * n_around
        for j in range(n_around):
            jn = (j + 1) % n_around
            tris.append([b0 + j, b0 + jn, b1 + jn])
            tris.append([b0 + j, b1 + jn, b1 + j])
    last = 1 + (len(rings) - 1) * n_around
    for j in range(n_around):
        tris.append([last + j, last + (j + 1) % n_around, top])
    return verts, np.asarray(tris, np.int32)


def fascia_shell(verts: np.ndarray, surface_tris: np.ndarray, gap: float = 0.001, thickness: float = 0.003):
    """A separate tet shell over an outward-oriented surface (the stand-in for an
    authored fascia asset of the ride mode): the surface vertices moved out by
    ``gap`` along their area-weighted normals, then extruded by ``thickness``
    as extrude_shell does (prisms of 3 tets, slivers dropped).  Shares no
    vertex with the muscle.  Returns (verts, tets)."""
    v = np.asarray(verts, np.float64)
    t = np.asarray(surface_tris, np.int64).reshape(-1, 3)
    fn = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    vn = np.zeros_like(v)
    for k in range(3):
        np.add.at(vn, t[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)
    moved = (v + gap * vn).astype(np.float32)
    shell, tets, _ = extrude_shell(moved, t, thickness)
    return shell.astype(np.float32), np.asarray(orient_tets(shell, tets), np.int32)


def capsule_sdf(x: np.ndarray, c: np.ndarray, axis: np.ndarray, half: float, r: float) -> np.ndarray:
    d = x - c
    t = np.clip(d @ axis, -half, half)
    return np.linalg.norm(d - t[..., None] * axis, axis=-1) - r


def humanv2_scene(seed: int = 0, n_muscles: int = 40, n_bones: int = 20, target_tets: int = 468_000,
                  fascia_tets: int = 70_000, fascia_thickness: float = 0.0015, tendon_frac: float = 0.05,
                  box=(0.7, 0.9, 0.7)) -> Scene:
    """Synthetic humanV2-scale muscle scene (~172.7k verts / ~535k tets at the
    defaults): ``n_muscles`` ellipsoids with length U(80,300) mm and radii
    U(10,40) mm, clipped 6-tet hex lattices, a ``fascia_thickness`` extruded
    shell over the first muscles' surfaces up to ``fascia_tets`` tets, and
    ``n_bones`` capsules (radius U(8,20) mm, length U(150,400) mm) on smooth
    rigid trajectories (rotation amplitude U(2.5,6.25) deg, translation
    amplitude U(5,20) mm)."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box)
    L = rng.uniform(0.080, 0.300, n_muscles)
    R1 = rng.uniform(0.010, 0.040, n_muscles)
    R2 = rng.uniform(0.010, 0.040, n_muscles)
    rots, cents, segs = [], [], []
    margin = 0.004
    for i in range(n_muscles):
        for _ in range(20000):
            Rm = _rand_rot(rng)
            c = rng.uniform(0, 1, 3) * box
            ax = Rm[:, 0]
            p0, p1 = c - ax * L[i] / 2, c + ax * L[i] / 2
            ri = max(R1[i], R2[i])
            if all(_seg_dist(p0, p1, q0, q1) > ri + rj + margin for (q0, q1, rj) in segs):
                break
        else:
            raise RuntimeError("could not place muscles; enlarge the box")
        rots.append(Rm)
        cents.append(c)
        segs.append((p0, p1, ri))
    bc, ba, bh, br = [], [], [], []
    for b in range(n_bones):
        for _ in range(20000):
            r = rng.uniform(0.008, 0.020)
            half = rng.uniform(0.150, 0.400) / 2
            c = rng.uniform(0, 1, 3) * box
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            p0, p1 = c - ax * half, c + ax * half
            ok = all(_seg_dist(p0, p1, q0, q1) > r + rj + 2 * margin for (q0, q1, rj) in segs)
            ok = ok and all(_seg_dist(p0, p1, bc[k] - ba[k] * bh[k], bc[k] + ba[k] * bh[k]) > r + br[k] + margin
                            for k in range(len(bc)))
            if ok:
                break
        else:
            raise RuntimeError("could not place bones; enlarge the box")
        bc.append(c)
        ba.append(ax)
        bh.append(half)
        br.append(r)
    bc, ba, bh, br = map(np.asarray, (bc, ba, bh, br))
    # lattice spacing for the muscle tet budget
    vol = 4.0 / 3.0 * np.pi * (L / 2) * R1 * R2
    h = (6.0 * vol.sum() / target_tets) ** (1.0 / 3.0)
    for _ in range(3):
        nt = sum(clipped_ellipsoid_lattice(L[i], R1[i], R2[i], h)[1].shape[0] for i in range(n_muscles))
        h *= (nt / target_tets) ** (1.0 / 3.0)
    verts, tets, tpart, vpart, vlocal_x, vlen = [], [], [], [], [], []
    off = 0
    for i in range(n_muscles):
        lv, lt = clipped_ellipsoid_lattice(L[i], R1[i], R2[i], h)
        wv = lv @ rots[i].T + cents[i]
        verts.append(wv)
        tets.append(lt + off)
        tpart.append(np.full(lt.shape[0], i))
        vpart.append(np.full(lv.shape[0], i))
        vlocal_x.append(lv[:, 0])
        vlen.append(np.full(lv.shape[0], L[i]))
        off += lv.shape[0]
    mverts = np.concatenate(verts)
    mtets = orient_tets(mverts, np.concatenate(tets))
    tpart = np.concatenate(tpart)
    vpart = np.concatenate(vpart)
    lx, lL = np.concatenate(vlocal_x), np.concatenate(vlen)
    xr = (lx + lL / 2) / lL
    tendon = ((xr < tendon_frac) | (xr > 1 - tendon_frac)).astype(np.float32)
    faces, opp = boundary_faces(mtets)
    surf = orient_faces_outward(mverts, faces, opp)
    # fascia shell over the first muscles' surfaces, up to the tet budget
    face_part = vpart[surf[:, 0]]
    chosen, acc = [], 0
    for i in range(n_muscles if fascia_tets > 0 else 0):  # fascia_tets <= 0: no shell
        nf = int((face_part == i).sum())
        if acc + 3 * nf > fascia_tets * 1.05 and chosen:
            continue
        chosen.append(i)
        acc += 3 * nf
        if acc >= fascia_tets * 0.95:
            break
    fsel = np.isin(face_part, chosen)
    if fsel.any():
        fverts, ftets, fsrc = extrude_shell(mverts, surf[fsel], fascia_thickness)
    else:
        fverts, ftets, fsrc = np.zeros((0, 3), np.float32), np.zeros((0, 4), np.int64), np.zeros(0, np.int64)
    nmv = mverts.shape[0]
    allv = np.concatenate([mverts, fverts]).astype(np.float32)
    ftets = orient_tets(allv, ftets + nmv)
    alltets = np.concatenate([mtets, ftets]).astype(np.int32)
    tet_part = np.concatenate([tpart, np.full(ftets.shape[0], -1)]).astype(np.int32)
    vert_part = np.concatenate([vpart, np.full(fverts.shape[0], -1)]).astype(np.int32)
    v_tendon = np.concatenate([tendon, np.zeros(fverts.shape[0], np.float32)])
    # fibers: each muscle's long axis with N(0, 10 deg) per-vertex noise
    fib = np.zeros((allv.shape[0], 3))
    for i in range(n_muscles):
        sel = np.nonzero(vpart == i)[0]
        ax = rots[i][:, 0]
        perp = np.cross(ax, rng.normal(size=(sel.shape[0], 3)))
        perp /= np.maximum(np.linalg.norm(perp, axis=1, keepdims=True), 1e-12)
        ang = np.deg2rad(rng.normal(0.0, 10.0, sel.shape[0]))
        fib[sel] = np.cos(ang)[:, None] * ax + np.sin(ang)[:, None] * perp
    fib[vert_part < 0] = [1.0, 0.0, 0.0]
    # two-bone binding: each muscle rides the bones nearest its two axial ends,
    # blended linearly along the axis (smooth within a muscle); fascia vertices
    # inherit the binding of the surface vertex they were extruded from
    end_bone = np.zeros((n_muscles, 2), np.int64)
    for i in range(n_muscles):
        ax = rots[i][:, 0]
        for k, sgn in enumerate((-1.0, 1.0)):
            e = cents[i] + sgn * ax * L[i] / 2
            end_bone[i, k] = int(np.argmin([capsule_sdf(e[None], bc[b], ba[b], bh[b], br[b])[0]
                                            for b in range(n_bones)]))
    mb = end_bone[vpart]
    mw = np.clip(xr, 0.0, 1.0)
    vert_bone = np.concatenate([mb, mb[fsrc]]).astype(np.int32)
    vert_bw = np.concatenate([mw, mw[fsrc]]).astype(np.float32)
    aniso = int(np.argmax(L * R1 * R2))
    # amplitudes that keep the bone-driven target field of every muscle
    # within stretches of 0.70..1.37 over frames 1-50 at the default scene
    traj = dict(rot_axis=rng.normal(size=(n_bones, 3)), rot_amp=np.deg2rad(rng.uniform(2.5, 6.25, n_bones)),
                rot_w=rng.uniform(0.05, 0.12, n_bones), rot_phase=rng.uniform(0, 2 * np.pi, n_bones),
                tr_dir=rng.normal(size=(n_bones, 3)), tr_amp=rng.uniform(0.005, 0.02, n_bones),
                tr_w=rng.uniform(0.05, 0.12, n_bones), tr_phase=rng.uniform(0, 2 * np.pi, n_bones))
    traj["tr_dir"] /= np.linalg.norm(traj["tr_dir"], axis=1, keepdims=True)
    traj["start_frame"] = 1
    return Scene(verts=allv, tets=alltets, tet_part=tet_part, vert_part=vert_part, v_tendon=v_tendon,
                 v_fiber=fib.astype(np.float32), surface_tris=surf.astype(np.int32), bone_center=bc, bone_axis=ba,
                 bone_half=bh, bone_radius=br, vert_bone=vert_bone, vert_bw=vert_bw, traj=traj, aniso_muscle=aniso,
                 muscle_rot=np.stack(rots), muscle_center=np.stack(cents), muscle_len=L,
                 meta=dict(seed=seed, h=h, n_muscle_verts=nmv, n_muscle_tets=mtets.shape[0],
                           n_fascia_tets=ftets.shape[0], fascia_muscles=chosen))


# --------------------------------------------------------------------------
# Coarse cage for the two-level multigrid


@dataclass
class Cage:
    """Per-muscle coarse hex cage (6 tets per cell) enclosing the fine muscle
    vertices, with the same arrays as the reference's baked cage npz
    (mg/mg.py:744-800): fine vertex -> coarse tet (cage_idx, -1 = not
    embedded) and barycentric uvw, and the Galerkin restriction
    (P^T P)^-1 stored per muscle block (minv_flat, blk_base, blk_dim,
    blk_matoff)."""
    coarse_pos: np.ndarray
    coarse_tet: np.ndarray
    cage_idx: np.ndarray
    uvw: np.ndarray
    minv_flat: np.ndarray
    blk_base: np.ndarray
    blk_dim: np.ndarray
    blk_matoff: np.ndarray
    mg_fine_nv: int
    lam: float = 0.0          # Tikhonov weight of the prior in the restriction


def _bary(p, a, b, c, d):
    T = np.stack([b - a, c - a, d - a], axis=-1)
    w = np.linalg.solve(T, (p - a)[..., None])[..., 0]
    return np.concatenate([(1.0 - w.sum(-1))[..., None], w], -1)


def build_cage(scene: "Scene", spacing: float = 0.016, rel_lam: float = 1e-3, operator: str = "tikhonov") -> Cage:
    """Coarse cage: for every muscle a ``spacing`` hex lattice in the muscle's
    local frame over the cells that hold its fine vertices; fascia vertices are
    not embedded.  ``operator`` picks the per-muscle restriction block:
    "pinv" the reference's pinv(P^T P, rcond=1e-8) (tools/gen_coarse_cage.py:221),
    "tikhonov" inv(P^T P + lam I) with lam = rel_lam x the median diagonal."""
    if operator not in ("tikhonov", "pinv"):
        raise ValueError(f"operator must be 'tikhonov' or 'pinv', got {operator!r}")
    nv = scene.verts.shape[0]
    cage_idx = np.full(nv, -1, np.int64)
    uvw = np.zeros((nv, 3))
    cpos_all, ctet_all, blocks = [], [], []
    voff = toff = 0
    x64 = scene.verts.astype(np.float64)
    for m in range(scene.muscle_rot.shape[0]):
        sel = np.nonzero(scene.vert_part == m)[0]
        R, c = scene.muscle_rot[m], scene.muscle_center[m]
        loc = (x64[sel] - c) @ R
        lo = loc.min(0) - 1e-9
        cell = np.floor((loc - lo) / spacing).astype(np.int64)
        dims = cell.max(0) + 1
        key = (cell[:, 0] * dims[1] + cell[:, 1]) * dims[2] + cell[:, 2]
        ucell, cell_of = np.unique(key, return_inverse=True)
        ci = ucell // (dims[1] * dims[2])
        cj = (ucell // dims[2]) % dims[1]
        ck = ucell % dims[2]
        gid = lambda i, j, k: (i * (dims[1] + 1) + j) * (dims[2] + 1) + k  # noqa: E731
        tets = hex_to_tets(lambda dx, dy, dz: gid(ci + dx, cj + dy, ck + dz))  # (6*ncell,4), perm-major
        used, tl = np.unique(tets, return_inverse=True)
        tl = tl.reshape(-1, 4)
        gi = used // ((dims[1] + 1) * (dims[2] + 1))
        gj = (used // (dims[2] + 1)) % (dims[1] + 1)
        gk = used % (dims[2] + 1)
        cl = lo + spacing * np.stack([gi, gj, gk], 1)
        cw = cl @ R.T + c
        ncell = ucell.shape[0]
        # the 6 tets of cell q are rows q + r*ncell
        best_w = np.full((sel.shape[0], 4), -np.inf)
        best_t = np.zeros(sel.shape[0], np.int64)
        for r in range(6):
            t = cell_of + r * ncell
            w = _bary(loc, cl[tl[t, 0]], cl[tl[t, 1]], cl[tl[t, 2]], cl[tl[t, 3]])
            better = w.min(1) > best_w.min(1)
            best_w[better] = w[better]
            best_t[better] = t[better]
        # keep only the coarse tets that embed a fine vertex, and their corners
        # (every kept corner then carries prolongation weight, so the Galerkin
        # restriction defines it)
        kept, best_t = np.unique(best_t, return_inverse=True)
        tl = tl[kept]
        usedv, tl = np.unique(tl, return_inverse=True)
        tl = tl.reshape(-1, 4)
        cw = cw[usedv]
        cage_idx[sel] = best_t + toff
        uvw[sel] = best_w[:, 1:]
        # Galerkin block (P^T P)^-1 over this muscle's coarse verts
        n = cw.shape[0]
        Pm = np.zeros((sel.shape[0], n))
        rows = np.repeat(np.arange(sel.shape[0]), 4)
        np.add.at(Pm, (rows, tl[best_t].reshape(-1)), best_w.reshape(-1))
        blocks.append(Pm.T @ Pm)
        cpos_all.append(cw)
        ctet_all.append(tl + voff)
        voff += n
        toff += tl.shape[0]
    coarse_pos = np.concatenate(cpos_all).astype(np.float32)
    coarse_tet = orient_tets(coarse_pos, np.concatenate(ctet_all)).astype(np.int32)
    # orient_tets may swap pts[0]/pts[1]; remap the barycentric weights to match
    raw = np.concatenate(ctet_all)
    swapped = raw[:, 0] != coarse_tet[:, 0]
    emb = cage_idx >= 0
    sw = np.zeros(nv, bool)
    sw[emb] = swapped[cage_idx[emb]]
    # uvw are the weights of pts[1..3]; weight of pts[0] is 1-u-v-w; swapping pts 0/1
    u_old = uvw[sw, 0].copy()
    w0_old = 1.0 - uvw[sw].sum(1)
    uvw[sw, 0] = w0_old
    del u_old
    # Restriction x_c = argmin |P x_c - x_f|^2 + lam |x_c - prior|^2: the
    # Galerkin least squares of the reference (pinv(P^T P), mg.py:770-800) with
    # a small Tikhonov weight toward the previous coarse state, so that cage
    # corners carrying almost no fine weight stay where they were instead of
    # amplifying FP32 noise (lam = rel_lam x median diagonal of P^T P).
    if operator == "pinv":
        lam = 0.0
        blocks = [np.linalg.pinv(B, rcond=1e-8) for B in blocks]
    else:
        lam = rel_lam * float(np.median(np.concatenate([np.diag(B) for B in blocks])))
        blocks = [np.linalg.inv(B + lam * np.eye(B.shape[0])) for B in blocks]
    blk_base, blk_dim, blk_matoff, flat = [], [], [], []
    off = base = 0
    for B in blocks:
        n = B.shape[0]
        blk_base += [base] * n
        blk_dim += [n] * n
        blk_matoff += [off] * n
        flat.append(B.reshape(-1))
        off += n * n
        base += n
    return Cage(coarse_pos=coarse_pos, coarse_tet=coarse_tet, cage_idx=cage_idx.astype(np.int32),
                uvw=uvw.astype(np.float32), minv_flat=np.concatenate(flat).astype(np.float32),
                blk_base=np.asarray(blk_base, np.int32), blk_dim=np.asarray(blk_dim, np.int32),
                blk_matoff=np.asarray(blk_matoff, np.int32), mg_fine_nv=nv, lam=lam)


# --------------------------------------------------------------------------
# Batched instances: many independent box muscles in one vertex set


@dataclass
class BatchScene(Scene):
    """``n_inst`` independent box muscles packed back to back (CSR offsets
    inst_vptr / inst_tptr into verts / tets), each placed in its own cell of
    a square grid in x-z, with two capsule bones at its two ends (bones 2i and
    2i+1), a 64^3-class SDF grid frame of its own (sdf_frame: origin xyz, h)
    and a piecewise-linear activation schedule (act_knots[i, k] at frame
    1 + k * knot_every)."""
    inst_vptr: np.ndarray | None = None
    inst_tptr: np.ndarray | None = None
    vert_inst: np.ndarray | None = None
    tet_inst: np.ndarray | None = None
    act_knots: np.ndarray | None = None
    knot_every: int = 8
    sdf_frame: np.ndarray | None = None
    sdf_res: int = 64

    @property
    def n_inst(self) -> int:
        return int(self.inst_vptr.shape[0] - 1)

    def instance_activation(self, frame: int) -> np.ndarray:
        """(n_inst,) activation of every instance at ``frame``: linear between
        knots, held at the last knot."""
        f = (float(frame) - 1.0) / float(self.knot_every)
        k = int(np.clip(np.floor(f), 0, self.act_knots.shape[1] - 2))
        u = float(np.clip(f - k, 0.0, 1.0))
        return ((1.0 - u) * self.act_knots[:, k] + u * self.act_knots[:, k + 1]).astype(np.float32)

    def activation(self, frame: int, start: int = 1, end: int = 50) -> np.ndarray:
        """Per-tet activation (user tet order) of the instance schedules."""
        return self.instance_activation(frame)[self.tet_inst]


def batched_box_scene(n_inst: int = 256, seed: int = 120, tets_lo: int = 2000, tets_hi: int = 60000,
                      spacing: float = 0.0025, jitter: float = 0.0002, pin_frac: float = 0.05,
                      n_knots: int = 8, knot_every: int = 8, sdf_res: int = 64) -> BatchScene:
    """``n_inst`` box muscles with tet counts log-uniform in [tets_lo, tets_hi]
    (square cross-section s x s hexes with s from an aspect a ~ U(3,5), length
    set by the drawn count; the default seed draws 3.50M tets in total), 2.5 mm
    spacing, U(-0.2, 0.2) mm jitter, fibers +z, the first/last ``pin_frac`` of
    each box's z extent pinned to the bone at that end.  Bones: capsules
    along x just beyond the end faces (radius 0.3 x the box width), on seeded
    smooth rigid paths (rotation amplitude U(3,8) deg about the capsule centre,
    translation amplitude U(2,6) mm), identity at frame 1."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(tets_lo), np.log(tets_hi), n_inst))
    aspect = rng.uniform(3.0, 5.0, n_inst)
    dims = []
    for c, a in zip(counts, aspect):
        s = max(2, int(round((c / (6.0 * a)) ** (1.0 / 3.0))))
        dims.append((s, s, max(4, int(round(c / (6.0 * s * s))))))
    ext = max(d[2] for d in dims) * spacing
    pitch = ext + 0.06
    side = int(np.ceil(np.sqrt(n_inst)))
    verts, tets, vptr, tptr, vinst, tinst, tendon, vbone, vbw = [], [], [0], [0], [], [], [], [], []
    bc, ba, bh, br, frames = [], [], [], [], []
    for i, (nx, ny, nz) in enumerate(dims):
        m = box_muscle(nx=nx, ny=ny, nz=nz, spacing=spacing, jitter=jitter, seed=seed * 100003 + i, pin_frac=pin_frac)
        off = np.array([(i % side) * pitch, 0.0, (i // side) * pitch], np.float32)
        v = m.verts + off
        z = v[:, 2]
        zr = (z - z.min()) / (z.max() - z.min())
        verts.append(v)
        tets.append(m.tets + vptr[-1])
        vptr.append(vptr[-1] + v.shape[0])
        tptr.append(tptr[-1] + m.tets.shape[0])
        vinst.append(np.full(v.shape[0], i))
        tinst.append(np.full(m.tets.shape[0], i))
        tendon.append(m.stopped.astype(np.float32))
        vbone.append(np.tile([2 * i, 2 * i + 1], (v.shape[0], 1)))
        vbw.append(np.clip((zr - pin_frac) / (1.0 - 2.0 * pin_frac), 0.0, 1.0))
        lo, hi = v.min(0).astype(np.float64), v.max(0).astype(np.float64)
        w = hi[0] - lo[0]
        r = 0.3 * w
        for zend in (lo[2] - r - 0.001, hi[2] + r + 0.001):  # just beyond the end faces
            bc.append([0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), zend])
            ba.append([1.0, 0.0, 0.0])
            bh.append(0.5 * w + r)
            br.append(r)
        margin = 3.0 * r + 0.012
        glo = lo - margin
        h = float((hi - lo + 2 * margin).max()) / (sdf_res - 1)
        frames.append([glo[0], glo[1], glo[2], h])
    verts = np.concatenate(verts).astype(np.float32)
    nb = 2 * n_inst
    traj = dict(rot_axis=rng.normal(size=(nb, 3)), rot_amp=np.deg2rad(rng.uniform(3.0, 8.0, nb)),
                rot_w=rng.uniform(0.05, 0.12, nb), rot_phase=rng.uniform(0, 2 * np.pi, nb),
                tr_dir=rng.normal(size=(nb, 3)), tr_amp=rng.uniform(0.002, 0.006, nb),
                tr_w=rng.uniform(0.05, 0.12, nb), tr_phase=rng.uniform(0, 2 * np.pi, nb), start_frame=1)
    traj["tr_dir"] /= np.linalg.norm(traj["tr_dir"], axis=1, keepdims=True)
    knots = rng.uniform(0.0, 1.0, (n_inst, n_knots)).astype(np.float32)
    knots[:, 0] = 0.0
    vinst = np.concatenate(vinst).astype(np.int32)
    tinst = np.concatenate(tinst).astype(np.int32)
    return BatchScene(
        verts=verts, tets=np.concatenate(tets).astype(np.int32), tet_part=tinst.copy(), vert_part=vinst.copy(),
        v_tendon=np.concatenate(tendon).astype(np.float32),
        v_fiber=np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (verts.shape[0], 1)),
        surface_tris=np.zeros((0, 3), np.int32), bone_center=np.asarray(bc), bone_axis=np.asarray(ba),
        bone_half=np.asarray(bh), bone_radius=np.asarray(br), vert_bone=np.concatenate(vbone).astype(np.int32),
        vert_bw=np.concatenate(vbw).astype(np.float32), traj=traj, aniso_muscle=-1,
        meta=dict(seed=seed, dims=dims, spacing=spacing),
        inst_vptr=np.asarray(vptr, np.int64), inst_tptr=np.asarray(tptr, np.int64), vert_inst=vinst, tet_inst=tinst,
        act_knots=knots, knot_every=knot_every, sdf_frame=np.asarray(frames, np.float32), sdf_res=sdf_res)


def batch_subset(sc: BatchScene, idx) -> BatchScene:
    """The instances ``idx`` of a batch as a batch of their own (CSR re-packed,
    bones 2i, 2i+1 and schedules carried along)."""
    idx = np.asarray(idx, np.int64)
    verts, tets, vptr, tptr = [], [], [0], [0]
    vsel_all, tsel_all, bones = [], [], []
    for j, i in enumerate(idx):
        v0, v1 = sc.inst_vptr[i], sc.inst_vptr[i + 1]
        t0, t1 = sc.inst_tptr[i], sc.inst_tptr[i + 1]
        vsel_all.append(np.arange(v0, v1))
        tsel_all.append(np.arange(t0, t1))
        tets.append(sc.tets[t0:t1] - v0 + vptr[-1])
        vptr.append(vptr[-1] + (v1 - v0))
        tptr.append(tptr[-1] + (t1 - t0))
        bones += [2 * i, 2 * i + 1]
    vs, ts, bones = np.concatenate(vsel_all), np.concatenate(tsel_all), np.asarray(bones)
    remap = np.full(2 * sc.n_inst, -1, np.int64)
    remap[bones] = np.arange(bones.shape[0])
    vinst = np.repeat(np.arange(idx.shape[0]), np.diff(vptr)).astype(np.int32)
    tinst = np.repeat(np.arange(idx.shape[0]), np.diff(tptr)).astype(np.int32)
    traj = {k: (v[bones] if isinstance(v, np.ndarray) and v.shape[:1] == (2 * sc.n_inst,) else v)
            for k, v in sc.traj.items()}
    return BatchScene(
        verts=sc.verts[vs], tets=np.concatenate(tets).astype(np.int32), tet_part=tinst.copy(), vert_part=vinst.copy(),
        v_tendon=sc.v_tendon[vs], v_fiber=sc.v_fiber[vs], surface_tris=np.zeros((0, 3), np.int32),
        bone_center=sc.bone_center[bones], bone_axis=sc.bone_axis[bones], bone_half=sc.bone_half[bones],
        bone_radius=sc.bone_radius[bones], vert_bone=remap[sc.vert_bone[vs]].astype(np.int32),
        vert_bw=sc.vert_bw[vs], traj=traj, aniso_muscle=-1, meta=dict(sc.meta, subset=idx.tolist()),
        inst_vptr=np.asarray(vptr, np.int64), inst_tptr=np.asarray(tptr, np.int64), vert_inst=vinst, tet_inst=tinst,
        act_knots=sc.act_knots[idx], knot_every=sc.knot_every, sdf_frame=sc.sdf_frame[idx], sdf_res=sc.sdf_res)


def shard_instances(tet_counts, world: int) -> list[list[int]]:
    """Greedy bin packing of instances over ``world`` ranks by tet count
    (largest first onto the lightest rank); each rank's list sorted."""
    order = np.argsort(-np.asarray(tet_counts), kind="stable")
    load = np.zeros(world, np.int64)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += int(tet_counts[i])
    return [sorted(x) for x in out]


def reseed_motion(sc: Scene, seed: int, n_frames: int = 64) -> Scene:
    """The same mesh with bone paths and a fiber activation schedule drawn
    from ``seed`` (amplitudes and frequencies from the same distributions as
    the scene's own; activation knots U(0,1) every 8 frames, 0 at frame 1)."""
    import dataclasses
    rng = np.random.default_rng(10_000 + int(seed))
    nb = sc.n_bones
    traj = dict(rot_axis=rng.normal(size=(nb, 3)), rot_amp=np.deg2rad(rng.uniform(2.5, 6.25, nb)),
                rot_w=rng.uniform(0.05, 0.12, nb), rot_phase=rng.uniform(0, 2 * np.pi, nb),
                tr_dir=rng.normal(size=(nb, 3)), tr_amp=rng.uniform(0.005, 0.02, nb),
                tr_w=rng.uniform(0.05, 0.12, nb), tr_phase=rng.uniform(0, 2 * np.pi, nb),
                start_frame=sc.traj.get("start_frame", 1))
    traj["tr_dir"] /= np.linalg.norm(traj["tr_dir"], axis=1, keepdims=True)
    knots = rng.uniform(0.0, 1.0, n_frames // 8 + 2).astype(np.float32)
    knots[0] = 0.0
    return dataclasses.replace(sc, traj=traj, act_sched=knots, meta=dict(sc.meta, motion_seed=int(seed)))


# arrays of a baked cage file, as the reference's cage baker writes them
# (tools/gen_coarse_cage.py:261) and its multigrid loads them (mg/mg.py:773-795)
CAGE_NPZ_KEYS = ("coarse_pos", "coarse_tet", "cage_idx", "uvw", "minv_flat", "blk_base", "blk_dim",
                 "blk_matoff", "mg_fine_nv")


def save_cage_npz(cage: Cage, path) -> None:
    """Write ``cage`` with the reference's cage-file keys plus ``lam`` (the
    Tikhonov weight its restriction blocks were inverted with; absent in the
    reference's files, whose blocks are pinv(P^T P), i.e. lam = 0)."""
    with open(path, "wb") as f:  # a file object keeps the name as given (no ".npz" appended)
        np.savez(f, coarse_pos=cage.coarse_pos.astype(np.float32), coarse_tet=cage.coarse_tet.astype(np.int32),
                 cage_idx=cage.cage_idx.astype(np.int32), uvw=cage.uvw.astype(np.float32),
                 minv_flat=cage.minv_flat.astype(np.float32), blk_base=cage.blk_base.astype(np.int32),
                 blk_dim=cage.blk_dim.astype(np.int32), blk_matoff=cage.blk_matoff.astype(np.int32),
                 mg_fine_nv=np.int64(cage.mg_fine_nv), lam=np.float64(cage.lam))


def load_cage_npz(path, n_verts: int) -> Cage:
    """Read a baked cage file (the reference's or ``save_cage_npz``'s).  Like
    the reference (mg/mg.py:774-779) it refuses a cage baked for another fine
    vertex count, and it checks that the block tables index inside the coarse
    vertex and Minv arrays, since the device restriction trusts them."""
    with np.load(path) as z:
        d = {k: z[k] for k in z.files}
    missing = [k for k in CAGE_NPZ_KEYS if k not in d]
    if missing:
        raise ValueError(f"cage file {path} lacks {missing}")
    nv = int(d["mg_fine_nv"])
    if nv != int(n_verts):
        raise ValueError(f"cage file {path} was built for fine NV={nv} but this scene has NV={int(n_verts)}")
    cage = Cage(coarse_pos=np.asarray(d["coarse_pos"], np.float32).reshape(-1, 3),
                coarse_tet=np.asarray(d["coarse_tet"], np.int32).reshape(-1, 4),
                cage_idx=np.asarray(d["cage_idx"], np.int32).reshape(-1),
                uvw=np.asarray(d["uvw"], np.float32).reshape(-1, 3),
                minv_flat=np.asarray(d["minv_flat"], np.float32).reshape(-1),
                blk_base=np.asarray(d["blk_base"], np.int32).reshape(-1),
                blk_dim=np.asarray(d["blk_dim"], np.int32).reshape(-1),
                blk_matoff=np.asarray(d["blk_matoff"], np.int32).reshape(-1),
                mg_fine_nv=nv, lam=float(d["lam"]) if "lam" in d else 0.0)
    nc, nt = cage.coarse_pos.shape[0], cage.coarse_tet.shape[0]
    if cage.cage_idx.shape[0] != nv or cage.uvw.shape[0] != nv:
        raise ValueError(f"cage file {path}: cage_idx/uvw must have one row per fine vertex ({nv})")
    if cage.coarse_tet.size and (cage.coarse_tet.min() < 0 or cage.coarse_tet.max() >= nc):
        raise ValueError(f"cage file {path}: coarse_tet indexes outside the {nc} coarse vertices")
    if cage.cage_idx.size and (cage.cage_idx.min() < -1 or cage.cage_idx.max() >= nt):
        raise ValueError(f"cage file {path}: cage_idx indexes outside the {nt} coarse tets")
    if not (cage.blk_base.shape[0] == cage.blk_dim.shape[0] == cage.blk_matoff.shape[0] == nc):
        raise ValueError(f"cage file {path}: blk_base/blk_dim/blk_matoff need one entry per coarse vertex")
    ends = cage.blk_matoff.astype(np.int64) + cage.blk_dim.astype(np.int64) ** 2
    if nc and (cage.blk_base.min() < 0 or (cage.blk_base.astype(np.int64) + cage.blk_dim).max() > nc
               or cage.blk_dim.min() < 1 or cage.blk_matoff.min() < 0 or ends.max() > cage.minv_flat.shape[0]):
        raise ValueError(f"cage file {path}: block table points outside the coarse vertices or minv_flat")
    return cage


def cage_for_config(scene: "Scene", cfg, operator: str = "tikhonov") -> Cage:
    """The multigrid cage a config asks for: ``coarse_npz_path`` names a baked
    cage file, which is loaded; a missing file is baked here (this package's
    lattice cage, ``mg_cage_spacing``) and written there, as the reference
    bakes a missing one on first use (mg/mg.py:759-772); without a path the
    lattice cage is built in memory."""
    import os
    spacing = float(cfg.get("mg_cage_spacing", 0.016))
    path = cfg.get("coarse_npz_path")
    if not path:
        return build_cage(scene, spacing=spacing, operator=operator)
    path = str(path)
    if not os.path.exists(path):
        cage = build_cage(scene, spacing=spacing, operator=operator)
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        save_cage_npz(cage, path)
    return load_cage_npz(path, scene.verts.shape[0])


def coarse_in_fine_embedding(fine_pos, fine_tet, coarse_pos, k: int = 16):
    """Coarse-in-fine embedding of the "c2f" state restriction
    (_build_c2f_embedding, mg/mg.py:903-938): for every coarse vertex, among
    the k fine rest tets with the nearest centroids, the one whose barycentric
    weights have the largest minimum (the enclosing tet when there is one,
    else the least extrapolating); weights ordered like the tet's corners,
    the last one 1 - the others.  Returns (tet [nc, 4] int32 fine ids,
    w [nc, 4] float32)."""
    from scipy.spatial import cKDTree
    fp = np.asarray(fine_pos, np.float64)
    ft = np.asarray(fine_tet, np.int64)
    cp = np.asarray(coarse_pos, np.float64)
    k = int(min(k, ft.shape[0]))
    _, cand = cKDTree(fp[ft].mean(1)).query(cp, k=k)
    cand = cand.reshape(cp.shape[0], k)
    best_w = np.zeros((cp.shape[0], 4))
    best_t = ft[cand[:, 0]].copy()
    best = np.full(cp.shape[0], -np.inf)
    for j in range(k):
        t = ft[cand[:, j]]
        d = fp[t[:, 3]]
        T = np.stack([fp[t[:, 0]] - d, fp[t[:, 1]] - d, fp[t[:, 2]] - d], axis=-1)
        w3 = np.linalg.solve(T, (cp - d)[..., None])[..., 0]
        w = np.concatenate([w3, (1.0 - w3.sum(1))[:, None]], axis=1)
        score = w.min(1)
        up = score > best
        best[up], best_w[up], best_t[up] = score[up], w[up], t[up]
    return best_t.astype(np.int32), best_w.astype(np.float32)
