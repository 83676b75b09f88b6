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


def test_squeeze_kernels_match_oracle():
    lib = capi.load()
    rng = np.random.default_rng(8)
    nf, nm = 4000, 6000
    f4 = _v4(rng.random((nf, 3)).astype(np.float32))
    t4 = _v4(rng.random((nm, 3)).astype(np.float32))
    m4 = _v4(rng.random((nm, 3)).astype(np.float32))
    m4[:, 3] = rng.uniform(0.5, 2.0, nm)
    follow = rng.integers(0, nm, nf).astype(np.int32)
    prev = _v4((t4[follow, :3] - rng.normal(scale=0.01, size=(nf, 3))).astype(np.float32))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    fd, pd, td = d(f4), d(prev), d(t4)
    assert lib.xpbd_fascia_advect(nf, p(d(follow)), p(td), p(pd), p(fd), None) == 0
    local = np.arange(0, nf, 7).astype(np.int32)
    cons = rng.integers(0, nm, local.size).astype(np.int32)
    off = _v4(rng.normal(scale=0.01, size=(local.size, 3)).astype(np.float32))
    assert lib.xpbd_fascia_anchor(local.size, p(d(local)), p(d(cons)), p(d(off)), p(td), p(fd), None) == 0
    pf = rng.integers(0, nf, 3000).astype(np.int32)
    pm = rng.permutation(nm)[:3000].astype(np.int32)  # distinct muscle vertices: atomics = sequential
    rest = rng.uniform(0.0, 0.5, 3000).astype(np.float32)
    comp = rng.uniform(0.0, 1e-6, 3000).astype(np.float32)
    md = d(m4)
    assert lib.xpbd_fascia_glue(3000, p(d(pf)), p(d(pm)), p(d(rest)), p(d(comp)), p(fd), p(md), C.c_float(1 / 240.0),
                                C.c_float(0.3), None) == 0
    torch.cuda.synchronize()
    of, op = O.fascia_advect(follow, t4, prev, f4)
    of = O.fascia_anchor(local, cons, off, t4, of)
    om = O.fascia_glue(pf, pm, rest, comp, of, m4, 1 / 240.0, 0.3)
    errs = [np.abs(fd.cpu().numpy() - of).max(), np.abs(pd.cpu().numpy()[:, :3] - op[:, :3]).max(),
            np.abs(md.cpu().numpy() - om).max()]
    print(f"squeeze kernels: |gpu - oracle| {errs}")
    assert max(errs) < 1e-6


def test_multigrid_with_fascia_squeeze_steps():
    from rlmusclev2_b200.mg import MultiGridSim, load_config
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["use_fascia"] = True
    cfg["fascia_mode"] = "squeeze"
    cfg["constraints"] += [
        {"type": "tetarapsvd", "name": "fascia_arap", "enable": True, "stiffness": 1.0e5, "rest_scale": 0.97},
        {"type": "volume", "name": "fascia_volume", "enable": True, "stiffness": 1.0e8},
        {"type": "glue", "name": "fascia_glue", "enable": True, "stiffness": 1.0e6, "stiffness_scale": 0.01,
         "iterations": 4},
        {"type": "anchor", "name": "fascia_anchor", "enable": True, "count": 128}]
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=0, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    assert sim.fascia.n_glue > 0 and sim.fascia.n_anchor >= 128
    f0 = sim.fascia.positions_np()
    for frame in range(1, 4):
        sim.set_fiber_activation(sc.activation(frame))
        sim.step_frame(frame)
    fp, mp = sim.fascia.positions_np(), sim.positions_np()
    assert np.isfinite(fp).all() and np.isfinite(mp).all()
    # the shell rides the skeleton: it moved with the targets, and stays near the muscle
    from scipy.spatial import cKDTree
    dist, _ = cKDTree(mp).query(fp)
    print(f"fascia squeeze: shell moved up to {np.abs(fp - f0).max():.4f} m, "
          f"max distance to the muscle {dist.max():.4f} m")
    assert dist.max() < 0.03
