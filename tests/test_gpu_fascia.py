"""Fascia ride mode on the GPU: xpbd_surface_bind / xpbd_surface_ride against
the oracle on the synthetic shell of a small scene (ties aside, as for the
bone binding), and MultiGridSim with use_fascia / fascia_mode="ride"."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.meshgen import fascia_shell, humanv2_scene

pytestmark = pytest.mark.gpu


def _v4(a):
    out = np.zeros((a.shape[0], 4), np.float32)
    out[:, :3] = a
    return out


def test_surface_bind_and_ride_match_oracle():
    lib = capi.load()
    sc = humanv2_scene(seed=2, n_muscles=3, n_bones=3, target_tets=6000, fascia_tets=0, box=(0.25, 0.25, 0.25))
    fv, _ = fascia_shell(sc.verts, sc.surface_tris, 0.001, 0.003)
    tris = np.ascontiguousarray(sc.surface_tris, np.int32)
    n = fv.shape[0]
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    q4, s4, td = d(_v4(fv)), d(_v4(sc.verts)), d(tris)
    face = torch.zeros(n, dtype=torch.int32, device="cuda")
    uv = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    gap = torch.zeros(n, dtype=torch.float32, device="cuda")
    ok = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert lib.xpbd_surface_bind(n, p(q4), sc.verts.shape[0], p(s4), tris.shape[0], p(td), C.c_float(0.05), p(face),
                                 p(uv), p(gap), p(ok), None) == 0
    torch.cuda.synchronize()
    of, ouv, ogap, ook = O.surface_bind(fv, sc.verts, tris, 0.05)
    gf, guv, ggap, gok = face.cpu().numpy(), uv.cpu().numpy(), gap.cpu().numpy(), ok.cpu().numpy()
    assert np.array_equal(gok, ook)
    same = gf == of
    print(f"surface bind: faces equal {same.mean():.4%}")
    # the shell's vertices sit on the surface vertices' normals, so many closest
    # points are surface corners shared by several faces (ties either side may
    # take); the closest distance must agree everywhere, the gap where the faces do
    assert same.mean() > 0.5

    def cpd(face, uv):
        A, B, Cc = sc.verts[tris[face, 0]], sc.verts[tris[face, 1]], sc.verts[tris[face, 2]]
        cp = uv[:, :1] * A + uv[:, 1:] * B + (1 - uv.sum(1, keepdims=True)) * Cc
        return np.linalg.norm(fv - cp, axis=1)
    m = gok == 1
    assert np.abs(cpd(gf, guv)[m] - cpd(of, ouv)[m]).max() < 1e-6
    assert np.abs(ggap[same & m] - ogap[same & m]).max() < 1e-6
    # ride on a moved muscle surface with the GPU's binding
    rng = np.random.default_rng(1)
    moved = (sc.verts + rng.normal(scale=0.001, size=sc.verts.shape)).astype(np.float32)
    bound = np.nonzero(gok)[0].astype(np.int32)
    out = d(_v4(fv))
    assert lib.xpbd_surface_ride(bound.size, p(d(bound)), p(d(gf[bound])), p(d(guv[bound])), p(d(ggap[bound])),
                                 p(d(_v4(moved))), p(td), p(out), None) == 0
    torch.cuda.synchronize()
    ref = O.surface_ride(bound, gf[bound], guv[bound], ggap[bound], moved, tris, fv)
    err = np.abs(out.cpu().numpy()[:, :3] - ref).max()
    print(f"surface ride: |gpu - oracle| {err:.2e}")
    assert err < 1e-6


def test_multigrid_with_fascia_ride_steps():
    from rlmusclev2_b200.mg import MultiGridSim, load_config
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["use_fascia"] = True
    cfg["fascia_mode"] = "ride"
    cfg["constraints"].append({"type": "snh", "name": "fascia_snh", "enable": True, "mu": 2.0e4, "lam": 1.0e6})
    cfg["constraints"].append({"type": "glue", "name": "fascia_glue", "enable": True, "iterations": 4})
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=0, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    assert sim.fascia is not None and sim.fascia.n_bound > 0.9 * sim.fascia.solver.n_verts
    for frame in range(1, 4):
        sim.set_fiber_activation(sc.activation(frame))
        sim.step_frame(frame)
    fp = sim.fascia.positions_np()
    mp = sim.positions_np()
    assert np.isfinite(fp).all() and np.isfinite(mp).all()
    # the shell stays on the muscle: every shell vertex within a few mm of the muscle surface
    from scipy.spatial import cKDTree
    dist, _ = cKDTree(mp[np.unique(sc.surface_tris)]).query(fp)
    print(f"fascia ride: bound {sim.fascia.n_bound}/{sim.fascia.solver.n_verts}, max distance to the muscle "
          f"surface vertices {dist.max():.4f} m")
    assert dist.max() < 0.02
