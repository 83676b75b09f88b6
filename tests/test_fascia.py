"""Fascia ride mode on the CPU: the synthetic shell is a valid tet mesh over
the muscle surface, and the oracle's bind + ride (fascia/fascia.py:130-176)
put an interior-bound vertex back where it was on the rest surface."""
import numpy as np

from oracle import oracle as O
from rlmusclev2_b200.meshgen import fascia_shell, humanv2_scene


def _scene():
    return humanv2_scene(seed=2, n_muscles=3, n_bones=3, target_tets=6000, fascia_tets=0, box=(0.25, 0.25, 0.25))


def test_shell_is_a_positive_tet_mesh_outside_the_muscle():
    sc = _scene()
    fv, ft = fascia_shell(sc.verts, sc.surface_tris, 0.001, 0.003)
    q = fv[ft].astype(np.float64)
    # positively oriented with the pt3 reference vertex, like the scene's muscle tets
    vol = np.linalg.det(np.stack([q[:, 0] - q[:, 3], q[:, 1] - q[:, 3], q[:, 2] - q[:, 3]], 1)) / 6
    assert (vol > 0).all() and ft.shape[0] > 2 * sc.surface_tris.shape[0]
    used = np.unique(sc.surface_tris)
    assert fv.shape[0] == 2 * used.shape[0]
    # inner layer 1 mm, outer 4 mm off the surface vertices
    d_in = np.linalg.norm(fv[: used.shape[0]] - sc.verts[used], axis=1)
    d_out = np.linalg.norm(fv[used.shape[0]:] - sc.verts[used], axis=1)
    np.testing.assert_allclose(d_in, 0.001, rtol=1e-3)
    np.testing.assert_allclose(d_out, 0.004, atol=1e-5)  # the outer layer follows the moved normals


def test_bind_then_ride_on_the_rest_surface():
    sc = _scene()
    fv, _ = fascia_shell(sc.verts, sc.surface_tris, 0.001, 0.003)
    face, uv, gap, ok = O.surface_bind(fv, sc.verts, sc.surface_tris, 0.05)
    assert ok.mean() > 0.99
    assert (np.abs(gap[ok == 1]) <= 0.05).all()
    bound = np.nonzero(ok)[0]
    back = O.surface_ride(bound, face[bound], uv[bound], gap[bound], sc.verts, sc.surface_tris, fv)
    inner = (uv[:, 0] > 1e-4) & (uv[:, 1] > 1e-4) & (uv.sum(1) < 1 - 1e-4)  # closest point inside its face
    sel = bound[inner[bound]]
    assert sel.size > 0
    assert np.abs(back[sel] - fv[sel]).max() < 1e-6


def test_squeeze_coupling_steps():
    """fascia_advect_bone / fascia_anchor_bone / solve_glue (fascia.py:45-125)."""
    rng = np.random.default_rng(4)
    nf, nm = 50, 80
    f4 = np.zeros((nf, 4), np.float32)
    f4[:, :3] = rng.random((nf, 3))
    t4 = np.zeros((nm, 4), np.float32)
    t4[:, :3] = rng.random((nm, 3))
    follow = rng.integers(0, nm, nf)
    prev = np.zeros((nf, 4), np.float32)
    prev[:, :3] = t4[follow, :3] - 0.01
    out, p2 = O.fascia_advect(follow, t4, prev, f4)
    np.testing.assert_allclose(out[:, :3], f4[:, :3] + 0.01, atol=1e-6)
    np.testing.assert_array_equal(p2[:, :3], t4[follow, :3])
    local, cons = np.arange(0, nf, 5), rng.integers(0, nm, 10)
    off = np.zeros((10, 4), np.float32)
    off[:, :3] = rng.normal(scale=0.01, size=(10, 3))
    snapped = O.fascia_anchor(local, cons, off, t4, f4)
    np.testing.assert_allclose(snapped[local, :3], t4[cons, :3] + off[:, :3], atol=1e-7)
    m4 = np.zeros((nm, 4), np.float32)
    m4[:, :3] = rng.random((nm, 3))
    m4[:, 3] = 1.0
    pf, pm = rng.integers(0, nf, 30), rng.permutation(nm)[:30]
    rest = (np.linalg.norm(f4[pf, :3] - m4[pm, :3], axis=1) * 0.7).astype(np.float32)
    moved = O.fascia_glue(pf, pm, rest, np.zeros(30, np.float32), f4, m4, 1.0 / 240.0, 1.0)
    np.testing.assert_allclose(np.linalg.norm(f4[pf, :3] - moved[pm, :3], axis=1), rest, rtol=1e-5)
