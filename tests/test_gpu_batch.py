"""Batched instances on the GPU: per-instance SDF bake, frames against the
oracle's batched program, persistent tile ranges against per-iteration
launches, and the full 256-instance (3.5M-tet) batch with the autotuner.

Frame gate as for the single scene: within the reference's FP32 run-to-run
gate of 1e-4 m or three times the oracle's own FP32/FP64 spread."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.batch import BatchSim
from rlmusclev2_b200.meshgen import batched_box_scene
from rlmusclev2_b200.mg import load_config
from tests._cases import bbox_diag

pytestmark = pytest.mark.gpu
CFG = "rlmusclev2_b200/configs/batched_256.json"
REF_ATOL = 1e-4


def _small(n=6, seed=3):
    cfg = load_config(CFG)
    cfg["demo"]["collision"]["sdf_res"] = 32
    sc = batched_box_scene(n_inst=n, seed=seed, tets_lo=800, tets_hi=4000, sdf_res=32)
    return cfg, sc


def test_batched_sdf_bake_matches_single_grid_and_oracle():
    cfg, sc = _small()
    sim = BatchSim(cfg, scene=sc)
    frame = 9
    sim.load_frame_targets(frame)
    sim.bone_collider.bake()
    sim.synchronize()
    got = sim.bone_collider.phi.cpu().numpy()
    T = sc.bone_transforms(frame).reshape(-1, 12).astype(np.float32)
    caps = np.concatenate([sc.bone_center, sc.bone_half[:, None], sc.bone_axis, sc.bone_radius[:, None]], 1)
    r = sc.sdf_res
    one = torch.empty((r, r, r), dtype=torch.float32, device=sim.device)
    bc = sim.bone_collider
    for i in range(sc.n_inst):
        fr = sc.sdf_frame[i].astype(np.float64)
        ref = O.sdf_bake((r, r, r), fr[:3], float(fr[3]), caps[2 * i:2 * i + 2], T[2 * i:2 * i + 2], bc.band, "f32")
        np.testing.assert_allclose(got[i], ref, atol=2e-6)
        s = capi.XpbdSdf()
        s.phi, s.nx, s.ny, s.nz = one.data_ptr(), r, r, r
        s.origin[:] = [float(x) for x in sc.sdf_frame[i, :3]]
        s.h = float(sc.sdf_frame[i, 3])
        capi.check(sim._lib.xpbd_sdf_bake_capsules(C.byref(s), 2, C.c_void_p(bc._caps.data_ptr() + 2 * 32 * i),
                                                   C.c_void_p(sim._bone_tr.data_ptr() + 2 * 48 * i),
                                                   C.c_float(bc.band), sim._sp))
        sim.synchronize()
        np.testing.assert_array_equal(one.cpu().numpy(), got[i])
    assert (got < 0).any()


def test_small_batch_frames_vs_oracle():
    cfg, sc = _small()
    sim = BatchSim(cfg, scene=sc)
    o32 = O.OracleBatchSim(cfg, sc, prec="f32")
    o64 = O.OracleBatchSim(cfg, sc, prec="f64")
    for frame in (1, 2, 3):
        sim.step_frame_inputs(frame)
        for o in (o32, o64):
            o.step_frame(frame)
        p = sim.positions_np()
        e64 = np.abs(p - o64.pos).max()
        spread = np.abs(o32.pos - o64.pos).max()
        moved = np.abs(o64.pos - sc.verts).max()
        print(f"batch frame {frame}: |gpu-o64| {e64:.3e} |gpu-o32| {np.abs(p - o32.pos).max():.3e} "
              f"spread {spread:.3e} moved {moved:.3e}")
        assert np.isfinite(p).all()
        assert e64 <= max(REF_ATOL, 3.0 * spread)
    assert moved > 1e-3
    assert sim.persistent_status() == 0


def test_persistent_tile_ranges_match_per_iteration():
    cfg, sc = _small(n=7, seed=5)
    sim = BatchSim(cfg, scene=sc)
    sim.step_frame_inputs(1)
    sim.load_frame_targets(4)
    sim._targets_kernel()
    sim.synchronize()
    per_grp = np.bincount(sim.layout.tile_group)
    sim._build_persist(int(per_grp.max()) + 1)
    assert len(sim._persist) > 2
    rng = np.random.default_rng(1)
    x = (sc.verts + rng.normal(scale=5e-4, size=sc.verts.shape)).astype(np.float32)
    sim.set_positions(x)
    start = sim._pos4.clone()
    for _ in range(6):
        sim._fused_iteration()
    ref = sim.positions_np()
    with torch.cuda.stream(sim._stream):
        sim._pos4.copy_(start)
    sim._fused_iterations(2)
    sim._fused_iterations(4)
    got = sim.positions_np()
    assert sim.persistent_status() == 0
    err, moved = np.abs(got - ref).max(), np.abs(ref - x).max()
    tol = 1e-5 * bbox_diag(sc.verts[sc.inst_vptr[0]:sc.inst_vptr[1]])
    print(f"{len(sim._persist)} ranges: max diff {err:.3e} moved {moved:.3e} tol {tol:.3e}")
    assert moved > 10 * tol and err <= tol


def test_full_batch_runs_and_autotunes():
    cfg = load_config(CFG)
    sim = BatchSim(cfg)
    assert sim.n_inst == 256 and 3.4e6 < sim.NT < 3.6e6
    sim.step_frame_inputs(1)
    best = sim.autotune(use_cache=False)
    print("autotune", best)
    for f in (2, 3):
        sim.step_frame_inputs(f)
    p = sim.positions_np()
    assert np.isfinite(p).all()
    act = sim.pin_active_np != 0
    d = np.linalg.norm(p[act] - sim.scene.targets(3)[act], axis=1)
    assert np.median(d) < 1e-5
    assert sim.persistent_status() == 0
    m = sim.metrics()
    assert m["n_nonfinite"] == 0
