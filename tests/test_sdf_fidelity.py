"""Fidelity of the bone push-out's grid SDF against the exact bone surface.

The reference pushes a vertex out of the bone along the surface normal by its
exact signed distance to the bone mesh (solve_mesh_contact_pos_kernel,
collision/sdf/kernel.py:122-170).  This project bakes the capsule bones of the
benchmark scene into a 256^3 FP32 grid over the scene's box once per frame
(the configuration's own choice) and pushes with the trilinear interpolant and
its gradient.  On the full-size config-2 scene at frame 1 (cell h = 4.19 mm,
bone radii 8-19 mm) this test measures the grid's distance error against the
exact capsule distance within one cell of the surface, the angle between the
grid gradient and the exact normal inside it, and the position difference
between a push-out by the grid and the exact push-out from the same points
up to one cell deep, with the penetration the grid push leaves.  The error is
the grid's resolution: trilinear interpolation of a distance field of
curvature 1/r errs by about h^2 / (8 r) (0.27 mm here); the figures are
recorded for the session summary and bounded in units of h.
"""
import numpy as np

from oracle import oracle as O
from rlmusclev2_b200.mg import load_config, scene_from_cfg

CFG = "rlmusclev2_b200/configs/humanv2_synth.json"


def _segments(sc, T):
    a = sc.bone_center - sc.bone_half[:, None] * sc.bone_axis
    b = sc.bone_center + sc.bone_half[:, None] * sc.bone_axis
    T = T.reshape(-1, 3, 4).astype(np.float64)
    aw = np.einsum("bij,bj->bi", T[:, :, :3], a) + T[:, :, 3]
    bw = np.einsum("bij,bj->bi", T[:, :, :3], b) + T[:, :, 3]
    return aw, bw, sc.bone_radius.astype(np.float64)


def _exact(x, aw, bw, r):
    """Signed distance to the union of capsules and its outward normal (float64)."""
    best = np.full(x.shape[0], np.inf)
    nrm = np.zeros_like(x)
    for a, b, rr in zip(aw, bw, r):
        ab = b - a
        t = np.clip(((x - a) @ ab) / (ab @ ab), 0.0, 1.0)
        v = x - (a + t[:, None] * ab)
        ln = np.linalg.norm(v, axis=1)
        d = ln - rr
        take = d < best
        best[take] = d[take]
        nrm[take] = v[take] / np.maximum(ln[take], 1e-30)[:, None]
    return best, nrm


def _trilinear(phi, origin, h, x):
    nz, ny, nx = phi.shape
    g = (x - origin) / h
    i = np.minimum(np.floor(g).astype(np.int64), np.array([nx - 2, ny - 2, nz - 2]))
    f = g - i
    p = phi.astype(np.float64)
    c = {(dx, dy, dz): p[i[:, 2] + dz, i[:, 1] + dy, i[:, 0] + dx] for dx in (0, 1) for dy in (0, 1) for dz in (0, 1)}
    fx, fy, fz = f[:, 0], f[:, 1], f[:, 2]
    c00 = c[0, 0, 0] + fx * (c[1, 0, 0] - c[0, 0, 0])
    c10 = c[0, 1, 0] + fx * (c[1, 1, 0] - c[0, 1, 0])
    c01 = c[0, 0, 1] + fx * (c[1, 0, 1] - c[0, 0, 1])
    c11 = c[0, 1, 1] + fx * (c[1, 1, 1] - c[0, 1, 1])
    c0 = c00 + fy * (c10 - c00)
    c1 = c01 + fy * (c11 - c01)
    val = c0 + fz * (c1 - c0)
    dx0 = (c[1, 0, 0] - c[0, 0, 0]) + fy * ((c[1, 1, 0] - c[0, 1, 0]) - (c[1, 0, 0] - c[0, 0, 0]))
    dx1 = (c[1, 0, 1] - c[0, 0, 1]) + fy * ((c[1, 1, 1] - c[0, 1, 1]) - (c[1, 0, 1] - c[0, 0, 1]))
    dy0 = (c[0, 1, 0] - c[0, 0, 0]) + fx * ((c[1, 1, 0] - c[1, 0, 0]) - (c[0, 1, 0] - c[0, 0, 0]))
    dy1 = (c[0, 1, 1] - c[0, 0, 1]) + fx * ((c[1, 1, 1] - c[1, 0, 1]) - (c[0, 1, 1] - c[0, 0, 1]))
    grad = np.stack([dx0 + fz * (dx1 - dx0), dy0 + fz * (dy1 - dy0), c1 - c0], 1) / h
    return val, grad


def test_grid_sdf_against_exact_capsules(parity_record):
    cfg = load_config(CFG)
    sc = scene_from_cfg(cfg)
    orc = O.OracleMultiGridSim(cfg, sc, prec="f32")
    T = sc.bone_transforms(1).astype(np.float32).reshape(-1, 12)
    r = orc.sdf_res
    phi = O.sdf_bake((r, r, r), orc.sdf_origin, orc.sdf_h, orc.caps, T, orc.band, "f32")
    h, band = orc.sdf_h, orc.band
    aw, bw, rad = _segments(sc, T)
    # random points of each capsule's bounding box grown by the band
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(np.minimum(a, b) - rr - band, np.maximum(a, b) + rr + band, size=(40000, 3))
                        for a, b, rr in zip(aw, bw, rad)])
    lo_box, hi_box = orc.sdf_origin, orc.sdf_origin + h * (r - 1)
    x = x[((x > lo_box + h) & (x < hi_box - h)).all(1)]
    d, n = _exact(x, aw, bw, rad)
    g, grad = _trilinear(phi, orc.sdf_origin, h, x)
    err = np.abs(g - d)
    gl = np.linalg.norm(grad, axis=1)
    ang = np.degrees(np.arccos(np.clip((grad * n).sum(1) / np.maximum(gl, 1e-30), -1, 1)))
    # the push-out acts on vertices that entered a bone during one substep:
    # the shell within one cell inside the surface
    shell = (d > -h) & (d < 0.0)
    near = np.abs(d) < h
    ins = shell & (d < -1e-6)
    xin = x[ins].astype(np.float32)
    pushed = xin.copy()
    O.sdf_push(pushed, np.ones(xin.shape[0], np.float32), phi, orc.sdf_origin, h, 0.0, -1.0, "f32")
    exact = x[ins] - n[ins] * d[ins][:, None]
    dpush = np.linalg.norm(pushed.astype(np.float64) - exact, axis=1)
    after, _ = _exact(pushed.astype(np.float64), aw, bw, rad)
    pen = np.maximum(0.0, -after)
    curv = h * h / (8.0 * rad.min())  # trilinear error scale of a field with curvature 1 / r_min
    parity_record("sdf_grid_vs_exact_capsules", h_m=h, band_m=band, r_min_m=rad.min(), h2_over_8r_m=curv,
                  near_samples=int(near.sum()), near_dist_err_max_m=err[near].max(),
                  near_dist_err_p99_m=np.percentile(err[near], 99), inside_dist_err_max_m=err[shell].max(),
                  inside_normal_err_p99_deg=np.percentile(ang[shell], 99), inside_normal_err_max_deg=ang[shell].max(),
                  push_samples=int(ins.sum()), push_diff_max_m=dpush.max(), push_diff_p99_m=np.percentile(dpush, 99),
                  residual_penetration_max_m=pen.max(), residual_penetration_p99_m=np.percentile(pen, 99))
    assert near.sum() > 20000 and ins.sum() > 10000
    # bounds: the measured figures with headroom, in units of the cell and of
    # the curvature error scale h^2 / (8 r_min)
    assert err[shell].max() <= 0.25 * h
    assert np.percentile(err[near], 99) <= 2.0 * curv
    assert np.percentile(ang[shell], 99) <= 20.0
    assert np.percentile(dpush, 99) <= 0.25 * h
    assert np.percentile(pen, 99) <= 0.15 * h
