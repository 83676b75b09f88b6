"""Two-level hpbd multigrid on the GPU vs the oracle (config 3's transfer path).

Per-operation gates from identical inputs: Galerkin restriction (FP32 block
solve; the oracle's FP32/FP64 spread of the same operator is ~1e-5 m, so the
gate is 5e-5 m), delta prolongation (1e-6 m), and one V-cycle including the
coarse ARAP sweeps (1e-5 x bbox diagonal on the coarse positions).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rlmusclev2_b200.meshgen import humanv2_scene
from rlmusclev2_b200.mg import MultiGridSim, load_config
from tests._cases import bbox_diag

pytestmark = pytest.mark.gpu
CFG = "rlmusclev2_b200/configs/humanv2_synth.json"


def _setup():
    cfg = load_config(CFG)
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["use_multigrid"] = True
    cfg["mg_coarse_iters"] = 2
    cfg["fine_iterations"] = 1
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    o64 = O.OracleMultiGridSim(cfg, sc, prec="f64")
    return cfg, sc, sim, o64


def _coarse_user(sim, t4):
    co = sim.mg.coarse
    a = t4[:, :3].cpu().numpy()
    out = np.empty_like(a)
    out[co.layout.perm] = a
    return out


def test_restrict_and_prolong_match_oracle():
    cfg, sc, sim, o64 = _setup()
    rng = np.random.default_rng(2)
    x = (sc.verts + rng.normal(scale=0.003, size=sc.verts.shape)).astype(np.float32)
    sim.set_positions(x)
    mg = sim.mg
    prior = _coarse_user(sim, mg.coarse._pos4)
    import ctypes as C
    from rlmusclev2_b200 import _capi as capi
    capi.check(sim._lib.xpbd_mg_restrict(C.byref(mg.g), C.c_void_p(sim._pos4.data_ptr()),
                                         C.c_void_p(mg.coarse._pos4.data_ptr()), C.c_void_p(mg.prev.data_ptr()),
                                         None, sim._sp))
    sim.synchronize()
    got = _coarse_user(sim, mg.coarse._pos4)
    ref = o64.restrict(x.astype(np.float64), prior.astype(np.float64))
    err = np.abs(got - ref).max()
    print(f"restrict max err {err:.3e}")
    assert err <= 5e-5
    np.testing.assert_array_equal(_coarse_user(sim, mg.prev), got)
    # prolong: perturb the coarse positions, compare the fine delta
    dc = rng.normal(scale=0.002, size=got.shape).astype(np.float32)
    newc = (got + dc).astype(np.float32)
    co = mg.coarse
    with torch.cuda.stream(sim._stream):
        co._pos4[:, :3] = torch.from_numpy(newc[co.layout.perm]).to(sim.device)
    capi.check(sim._lib.xpbd_mg_prolong_delta(C.byref(mg.g), C.c_void_p(co._pos4.data_ptr()),
                                              C.c_void_p(mg.prev.data_ptr()), C.c_void_p(sim._pos4.data_ptr()),
                                              None, None, sim._sp))
    fine = sim.positions_np()
    d = (newc.astype(np.float64) - got.astype(np.float64))
    e, w, t = o64.mg_emb, o64.mg_w, o64.mg_t
    expect = x.astype(np.float64).copy()
    expect[e] += sum(w[:, k:k + 1] * d[t[:, k]] for k in range(4))
    perr = np.abs(fine - expect).max()
    print(f"prolong max err {perr:.3e}")
    assert perr <= 1e-6


def test_vcycle_from_identical_state():
    cfg, sc, sim, o64 = _setup()
    frame = 3
    o64.target, _ = o64.targets(frame)
    o64.mg_target = o64.restrict(o64.target, o64.mg_target)
    sim.load_frame_targets(frame)
    sim._targets_kernel()
    sim.mg.refresh_target()
    rng = np.random.default_rng(4)
    x = (sc.verts + rng.normal(scale=0.002, size=sc.verts.shape)).astype(np.float32)
    sim.set_positions(x)
    o64.pos[:] = x
    sim.mg.vcycle(pin_fine=False)
    o64.vcycle()
    got = sim.positions_np()
    cg = _coarse_user(sim, sim.mg.coarse._pos4)
    tol = 1e-5 * bbox_diag(sc.verts)
    ce = np.abs(cg - o64.mg.pos).max()
    fe = np.abs(got - o64.pos).max()
    moved = np.abs(o64.pos - x).max()
    print(f"vcycle coarse err {ce:.3e} fine err {fe:.3e} moved {moved:.3e} tol {tol:.3e}")
    assert moved > 10 * tol
    assert ce <= tol + 5e-5 and fe <= tol + 5e-5


def test_mg_frames_run_and_stay_finite():
    cfg, sc, sim, o64 = _setup()
    o32 = O.OracleMultiGridSim(cfg, sc, prec="f32")
    for frame in (1, 2, 3):
        sim.set_fiber_activation(sc.activation(frame))
        sim.step_frame(frame)
        o32.step_frame(frame)
        o64.step_frame(frame)
    p = sim.positions_np()
    spread = np.abs(o32.pos - o64.pos).max()
    err = np.abs(p - o64.pos).max()
    print(f"mg frames: |gpu-o64| {err:.3e}  oracle FP32/FP64 spread {spread:.3e}")
    assert np.isfinite(p).all()
    assert err <= max(1e-4, 3.0 * spread)


def test_projection_mode_frames_vs_oracle():
    """mg_mode="projection" (mg.py:1263-1320): every substep the embedded fine
    vertices restart from the prolonged restricted bone target.  Three frames on
    the small scene without the skip threshold, against the FP64 oracle at three
    times the FP32 oracle's distance (max and p99)."""
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth_mg_dcd.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["demo"]["self_collision"]["method"] = "none"
    cfg["mg_mode"] = "projection"
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    sim._prm.arap_skip_ssq = -1.0
    o32 = O.OracleMultiGridSim(cfg, sc, prec="f32")
    o64 = O.OracleMultiGridSim(cfg, sc, prec="f64")
    tol = 1e-5 * bbox_diag(sc.verts)
    O.set_arap_skip(-1.0)
    try:
        for frame in (1, 2, 3):
            sim.set_fiber_activation(sc.activation(frame))
            sim.step_frame(frame)
            o32.step_frame(frame)
            o64.step_frame(frame)
            p = sim.positions_np()
            d = np.abs(p - o64.pos).max(1)
            spr = np.abs(o32.pos - o64.pos).max(1)
            print(f"projection frame {frame}: |gpu-o64| max {d.max():.3e} p99 {np.percentile(d, 99):.3e}; "
                  f"|o32-o64| max {spr.max():.3e}")
            assert np.isfinite(p).all()
            assert d.max() <= max(tol, 3.0 * spr.max())
            assert np.percentile(d, 99) <= max(tol, 3.0 * np.percentile(spr, 99))
    finally:
        O.set_arap_skip(0.0)
    assert np.abs(o64.pos - sc.verts).max() > 100 * tol


@pytest.mark.parametrize("restrict_mode,sync", [("galerkin", "galerkin"), ("none", "galerkin"), ("direct", "c2f")])
def test_restrict_modes_frames_vs_oracle(restrict_mode, sync):
    """Step 1 of the V-cycle by mg_restrict_mode / mg_sync_restrict
    (mg.py:224-246, 992-1012): the restricted bone target copied in, the coarse
    left on its own state, and the coarse-in-fine readout.  Three frames on the
    small scene without the skip threshold, against the FP64 oracle at three
    times the FP32 oracle's distance (max and p99)."""
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth_mg_dcd.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["demo"]["self_collision"]["method"] = "none"
    cfg["mg_restrict_mode"], cfg["mg_sync_restrict"] = restrict_mode, sync
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    # no skip threshold on either level: with "none" the cage relaxes across
    # frames, and the threshold then leaves out (and uncounts) nearly rigid tets
    sim._prm.arap_skip_ssq = -1.0
    sim.mg.coarse._prm.arap_skip_ssq = -1.0
    o32 = O.OracleMultiGridSim(cfg, sc, prec="f32")
    o64 = O.OracleMultiGridSim(cfg, sc, prec="f64")
    tol = 1e-5 * bbox_diag(sc.verts)
    O.set_arap_skip(-1.0)
    try:
        for frame in (1, 2, 3):
            sim.set_fiber_activation(sc.activation(frame))
            sim.step_frame(frame)
            o32.step_frame(frame)
            o64.step_frame(frame)
            p = sim.positions_np()
            d = np.abs(p - o64.pos).max(1)
            spr = np.abs(o32.pos - o64.pos).max(1)
            print(f"{restrict_mode}/{sync} frame {frame}: |gpu-o64| max {d.max():.3e} p99 "
                  f"{np.percentile(d, 99):.3e}; |o32-o64| max {spr.max():.3e}")
            assert np.isfinite(p).all()
            assert d.max() <= max(tol, 3.0 * spr.max())
            assert np.percentile(d, 99) <= max(tol, 3.0 * np.percentile(spr, 99))
    finally:
        O.set_arap_skip(0.0)
