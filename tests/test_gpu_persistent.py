"""The persistent multi-iteration pass (xpbd_iterate_persistent) against the
oracle and against the per-iteration launches it replaces.

One launch of n iterations must equal n x (tile pass + boundary finish): the
same Jacobi rounds, with tile vertices held in shared memory and boundary sums
through the three-slot ring.  Gates: against the FP32 oracle after 1 and 3
iterations on the mixed-constraint problem (damped volume and SNH, aniso,
attach: the damped constraint-set instance) at 1e-5 x bbox diagonal; against
the per-iteration path after 20 iterations of the synthetic humanV2 scene
(ARAP, aniso, belly attach, tendon pins: the light instance) at 1e-5 x bbox
diagonal, split over two launches to cross the ring phase; barrier status
clean throughout.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from rlmusclev2_b200.engine import XpbdSolver
from rlmusclev2_b200.mg import MultiGridSim, load_config
from rlmusclev2_b200.meshgen import humanv2_scene
from tests._cases import bbox_diag
from tests.test_gpu_parity import _mixed_problem, _oracle_table

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_iters", [1, 3])
def test_mixed_constraints_vs_oracle(n_iters):
    verts, tets, table, mass, vf, act, tendon, deformed, prev = _mixed_problem()
    kw = dict(dt=1.0 / 240.0, contraction_ratio=0.4, fiber_stiffness_scale=3.0)
    sim = XpbdSolver(verts, tets, table, mass=mass, v_fiber=vf, tet_tendonmask=tendon, device="cuda:0",
                     tile_tets=64, **kw)
    assert sim._persist_fits and sim.layout.n_tiles > 1
    sim.set_activation(act)
    sim.set_positions(prev, also_prev=True)
    sim.set_positions(deformed)
    _, B, _, _ = O.precompute_rest(verts, tets, 1060.0, "f32")
    o = O.OracleSolver(verts, tets, _oracle_table(table), mass, np.zeros(len(verts), np.int32), B,
                       gravity_vec=(0, 0, 0), v_fiber=vf, activation=act, tendonmask=tendon, prec="f32", **kw)
    o.pos[:] = deformed
    o.pprev[:] = prev
    for _ in range(n_iters):
        o.project()
        o.apply_dP()
    sim._fused_iterations(n_iters)
    got = sim.positions_np()
    assert sim.persistent_status() == 0
    tol = 1e-5 * bbox_diag(verts)
    err = np.abs(got - o.pos).max()
    moved = np.abs(o.pos - deformed).max()
    print(f"persistent n={n_iters}: |gpu-o32| {err:.3e} moved {moved:.3e} tol {tol:.3e}")
    assert moved > 10 * tol
    assert err <= tol


def test_humanv2_small_matches_per_iteration_path():
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    assert sim._persist_fits
    frame = 6
    sim.set_fiber_activation(sc.activation(frame))
    sim.load_frame_targets(frame)
    sim._targets_kernel()
    sim.synchronize()
    rng = np.random.default_rng(5)
    x = (sc.verts + rng.normal(scale=0.001, size=sc.verts.shape)).astype(np.float32)
    sim.set_positions(x)
    start = sim._pos4.clone()
    for _ in range(20):
        sim._fused_iteration()
    ref = sim.positions_np()
    with torch.cuda.stream(sim._stream):
        sim._pos4.copy_(start)
    sim._fused_iterations(7)
    sim._fused_iterations(13)
    got = sim.positions_np()
    assert sim.persistent_status() == 0
    tol = 1e-5 * bbox_diag(sc.verts)
    err = np.abs(got - ref).max()
    moved = np.abs(ref - x).max()
    print(f"persistent 7+13 vs 20 per-iteration: max diff {err:.3e} moved {moved:.3e} tol {tol:.3e}")
    assert moved > 10 * tol
    assert err <= tol
    assert int(sim._psync[2].item()) == 20 % 3


def test_fixed_point_range_check_flags_oversized_scale():
    """The tile passes sum corrections as round(d x acc_scale) in 32-bit
    integers.  With the library's scale for the mesh the range check stays
    clean; with a scale 2^20 times too large every sizeable correction leaves
    the safe range and the status word reports it (integer arithmetic only:
    the sums wrap, nothing faults)."""
    from rlmusclev2_b200 import _capi as capi
    verts, tets, table, mass, vf, act, tendon, deformed, prev = _mixed_problem()
    kw = dict(dt=1.0 / 240.0, contraction_ratio=0.4, fiber_stiffness_scale=3.0)
    sim = XpbdSolver(verts, tets, table, mass=mass, v_fiber=vf, tet_tendonmask=tendon, device="cuda:0",
                     tile_tets=64, **kw)
    sim.set_activation(act)
    sim.set_positions(prev, also_prev=True)
    sim.set_positions(deformed)
    sim._fused_iterations(2)
    assert sim.persistent_status() == 0
    sim._prm.acc_scale = sim._prm.acc_scale * 2.0 ** 20
    sim.set_positions(deformed)
    sim._fused_iterations(1)
    assert sim.persistent_status() & capi.STATUS_ACC_RANGE


@pytest.mark.parametrize("base", [0, 1])
def test_tile_pass_with_l2_prefetch_is_bit_identical(base):
    """tile_variant bit 5 only adds a bulk L2 prefetch of each tile's tet
    streams: the per-iteration pass gives the same positions bit for bit, at
    either CTAs-per-SM choice (bit 0)."""
    variant = base | 32
    verts, tets, table, mass, vf, act, tendon, deformed, prev = _mixed_problem()
    kw = dict(dt=1.0 / 240.0, contraction_ratio=0.4, fiber_stiffness_scale=3.0)
    out = []
    for tv in (base, variant):
        sim = XpbdSolver(verts, tets, table, mass=mass, v_fiber=vf, tet_tendonmask=tendon, device="cuda:0",
                         tile_tets=64, **kw)
        sim._prm.tile_variant = tv
        sim.set_activation(act)
        sim.set_positions(prev, also_prev=True)
        sim.set_positions(deformed)
        for _ in range(3):
            sim._fused_iteration()
        out.append(sim.positions_np())
    assert np.array_equal(out[0], out[1])
    assert np.abs(out[0] - deformed).max() > 0


@pytest.mark.parametrize("case", ["tangled", "flat"])
def test_deferred_svd_pass_is_bit_identical(case):
    """tile_variant bit 6 moves the tets whose rotation needs the SVD to a
    pass after the tile's loop: the per-iteration and the persistent passes
    give the same positions bit for bit.  "tangled": a jitter of 40 % of an
    edge inverts many tets (56 of 384); "flat": every tet squashed to a
    millionth of its height, so the one tile (all 384 tets) defers more than
    the list's 128 and the rest run in place."""
    verts, tets, table, mass, vf, act, tendon, deformed, prev = _mixed_problem()
    rng = np.random.default_rng(7)
    if case == "tangled":
        deformed = verts + rng.normal(scale=0.004, size=verts.shape).astype(np.float32)
    else:
        deformed = (verts * np.array([1.0, 1.0, 1e-6], np.float32)).astype(np.float32)
    kw = dict(dt=1.0 / 240.0, contraction_ratio=0.4, fiber_stiffness_scale=3.0)
    for persistent in (False, True):
        out = []
        for tv in (0, 64):
            sim = XpbdSolver(verts, tets, table, mass=mass, v_fiber=vf, tet_tendonmask=tendon, device="cuda:0",
                             tile_tets=512 if case == "flat" else 64, **kw)
            sim._prm.tile_variant = tv
            sim.set_activation(act)
            sim.set_positions(prev, also_prev=True)
            sim.set_positions(deformed)
            if persistent:
                sim._fused_iterations(3)
                assert sim.persistent_status() == 0
            else:
                for _ in range(3):
                    sim._fused_iteration()
            out.append(sim.positions_np())
        assert np.isfinite(out[0]).all()
        assert np.array_equal(out[0], out[1]), (case, persistent)
        assert np.abs(out[0] - deformed).max() > 0
