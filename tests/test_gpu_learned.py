"""The learned coarse warm start on the GPU: the feature kernel against a
host restatement, the cage-level fallback, and what the committed trained
network gains over the plain solver on a held-out motion seed (config 3's
mesh and cage, 20 Jacobi iterations per substep)."""
import numpy as np
import pytest
import torch

from rlmusclev2_b200 import learned as LW
from rlmusclev2_b200.meshgen import humanv2_scene, reseed_motion
from rlmusclev2_b200.mg import MultiGridSim

pytestmark = pytest.mark.gpu


def _small():
    cfg = LW.learned_config()
    cfg["demo"]["collision"]["sdf_res"] = 64
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    return sim, LW.LearnedWarmStart(sim)


def _lib_to_cage(ws, t4):
    lib = ws._lib_d.cpu().numpy()
    return t4[:, :3].cpu().numpy()[lib]


def test_features_match_host_restatement():
    sim, ws = _small()
    ws.reset(reseed_motion(sim.scene, 7))
    for f in (1, 2, 3):
        ws.frame(f, 5, learned=False)
    ws.begin_frame(4)
    ws.predict(0)
    ws.features()
    sim.synchronize()
    X = ws.net.X[:ws.nc].float().cpu().numpy()
    Xt = ws.net.Xt[:, :ws.nc].float().cpu().numpy()
    np.testing.assert_array_equal(X, Xt.T)
    cp, cq = _lib_to_cage(ws, ws.mg.prev), _lib_to_cage(ws, ws._cprev)
    crest, ctgt = _lib_to_cage(ws, ws._c0), _lib_to_cage(ws, ws.mg.pin4)
    st = LW._cage_static(sim)
    d = 1000.0 * (cp - cq)
    ref = np.zeros((ws.nc, 64))
    ref[:, 0:3] = d
    ref[:, 3] = sim.scene.muscle_activation(4)[st["owner"]]
    rel = LW.bone_relative(sim.scene, 4)
    v = rel[st["cbone"][:, 0]] + st["cw"][:, None] * (rel[st["cbone"][:, 1]] - rel[st["cbone"][:, 0]])
    v = v.reshape(-1, 3, 4)
    ref[:, 4:13] = 10.0 * (v[:, :, :3] - np.eye(3)).reshape(-1, 9)
    ref[:, 13:16] = 100.0 * v[:, :, 3]
    for q in range(6):
        k = st["nbr"][:, q]
        ref[:, 16 + 3 * q:19 + 3 * q] = np.where((k >= 0)[:, None], d[np.maximum(k, 0)] - d, 0.0)
    ref[:, 34:37] = 1000.0 * (cp - crest)
    ref[:, 37:40] = 1000.0 * (ctgt - cp)
    ref[:, 40:] = st["stat"]
    # BF16 storage: 3 significant digits, plus FP32 rounding of mm-scaled differences
    np.testing.assert_allclose(X, ref, rtol=1e-2, atol=2e-3)
    assert (st["nbr"] >= 0).mean() > 0.5


def test_fallback_drops_a_bad_correction_and_keeps_a_good_one():
    sim, ws = _small()
    ws.reset(reseed_motion(sim.scene, 9))
    ws.frame(1, 5, learned=False)
    ws.begin_frame(2)
    ws.predict(0)
    sim.synchronize()  # the clone runs on torch's current stream, not the engine's
    x_pred = sim._pos4.clone()
    # a network with a large random output layer: centimetre-scale non-rigid
    # cage corrections raise the cage's ARAP residual and are dropped (a rigid
    # shift would not change that residual)
    with torch.cuda.stream(ws.net.stream):
        ws.net.W[4].normal_(0.0, 50.0)
    ws.net.refresh_copies()
    ws.set_norm(None, 1.0)
    ws.features()
    ws.warm_start(fallback=True)
    sim.synchronize()
    assert int(ws.fallbacks.item()) == 1
    torch.testing.assert_close(sim._pos4, x_pred, rtol=0, atol=0)
    # a zero correction is kept (no fallback) and leaves x_pred unchanged up to the re-pin
    with torch.cuda.stream(ws.net.stream):
        ws.net.W[4].zero_()
        ws.net.b[4].zero_()
    ws.net.refresh_copies()
    ws.features()
    ws.warm_start(fallback=True)
    sim.synchronize()
    assert int(ws.fallbacks.item()) == 1
    assert float((sim._pos4 - x_pred).abs().max()) < 1e-7


def test_trained_network_gains_over_plain():
    """Held-out seed 41, frames 1-4: with the committed weights, the largest
    per-frame max error against the 200-iteration solve after 20 iterations
    is lower for the learned warm start than for the plain start."""
    sim = MultiGridSim(LW.learned_config())
    ws = LW.LearnedWarmStart(sim)
    meta = LW.load_weights(ws)
    err, rms = LW.evaluate(ws, [41], 4, [20])
    p = err["plain"][20].reshape(-1, sim.nsubsteps).max(1)
    q = err["learned"][20].reshape(-1, sim.nsubsteps).max(1)
    print(f"weights {meta}; per-frame max error plain {np.round(p, 3)} learned {np.round(q, 3)} mm; "
          f"rms plain {rms['plain'][20].mean():.4f} learned {rms['learned'][20].mean():.4f} mm")
    assert q[1:].sum() < 0.85 * p[1:].sum()


def test_residual_checked_fallback_takes_the_plain_solve():
    """fallback="residual": a network with a large random output layer gives
    a warm start whose post-iteration residual is above the plain solver's, so
    the substep ends on the plain solve from x_pred, bit for bit, and the
    choice is counted; with a zero network (no correction) the learned result
    is kept, and it equals the plain one."""
    sim, ws = _small()
    ws.reset(reseed_motion(sim.scene, 9))
    ws.frame(1, 5, learned=False)
    ws.begin_frame(2)
    ws.predict(0)
    sim.synchronize()  # clones run on torch's current stream, not the engine's
    x_pred = sim._pos4.clone()
    ws.iterate(4)
    sim.synchronize()
    x_plain = sim._pos4.clone()
    with torch.cuda.stream(sim._stream):
        sim._pos4.copy_(x_pred)
    with torch.cuda.stream(ws.net.stream):
        ws.net.W[4].normal_(0.0, 50.0)
    ws.net.refresh_copies()
    ws.set_norm(None, 1.0)
    ws.plain_taken.zero_()
    ws.plain_checked(4)
    sim.synchronize()
    assert int(ws.plain_taken.item()) == 1
    torch.testing.assert_close(sim._pos4, x_plain, rtol=0, atol=0)
    with torch.cuda.stream(ws.net.stream):
        ws.net.W[4].zero_()
        ws.net.b[4].zero_()
    ws.net.refresh_copies()
    with torch.cuda.stream(sim._stream):
        sim._pos4.copy_(x_pred)
    ws.plain_checked(4)
    sim.synchronize()
    assert int(ws.plain_taken.item()) == 1
    assert float((sim._pos4 - x_plain).abs().max()) < 1e-6
