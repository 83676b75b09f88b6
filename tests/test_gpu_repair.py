"""SVD inversion repair (XpbdEngine.repair_inverted_tets, engine.py:831-856)
on the GPU against the oracle: a box muscle squashed to a tenth of its height
along z (singular values ~0.1 below repair_sigma_min = 0.3) and one with a
layer of inverted tets, stepped with the repair in the finalize phase."""
import numpy as np
import pytest

from oracle import oracle as O
from rlmusclev2_b200 import MuscleSim
from rlmusclev2_b200.meshgen import box_muscle
from tests._cases import bbox_diag

pytestmark = pytest.mark.gpu
CONS = [{"type": "tetarapsvd", "name": "arap", "compliance": 1e-7},
        {"type": "volume", "name": "volume", "compliance": 0.0}]
KW = dict(dts=1.0 / 24.0, num_substeps=10, density=1060.0, veldamping=0.02, gravity=-9.8)


def _pair(start, alpha, iters, sigma_min):
    m = box_muscle()
    sim = MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS, device="cuda:0",
                                    stopped=m.stopped, **KW)
    sim.repair_alpha, sim.repair_iters, sim.repair_sigma_min = alpha, iters, sigma_min
    orc = O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS, stopped=m.stopped,
                            repair_alpha=alpha, repair_iters=iters, repair_sigma_min=sigma_min, prec="f32", **KW)
    sim.set_positions(start, also_prev=True)
    orc.pos[:] = start
    orc.pprev[:] = start
    return m, sim, orc


def _squashed(m):
    c = m.verts.mean(0)
    return (c + (m.verts - c) * np.array([1.0, 1.0, 0.1], np.float32)).astype(np.float32)


def test_clamp_pass_matches_oracle():
    """One repair call from the squashed state (no constraint step between)."""
    m = box_muscle()
    start = _squashed(m)
    _, sim, orc = _pair(start, 1.0, 2, 0.3)
    sim.repair_inverted_tets()
    orc.svd_clamp(0.3, 1.0, 2)
    p = sim.positions_np()
    moved = np.abs(orc.pos - start).max()
    assert moved > 1e-4
    # float atomics add the per-vertex sums in any order: rounding level
    assert np.abs(p - orc.pos).max() <= 1e-6 * max(1.0, float(np.abs(start).max()))
    assert np.array_equal(p[m.stopped != 0], start[m.stopped != 0])


@pytest.mark.parametrize("case", ["squashed", "inverted"])
def test_steps_with_repair_match_oracle(case):
    """Two frames with the repair in every substep.  Both starts are violent (the
    squashed box re-expands through inverted states, the mirrored layer unfolds),
    so the FP32 and FP64 oracles themselves part by 3e-5 m and by millimetres;
    the GPU is gated against the FP64 oracle at three times that spread (max and
    p99), and its inverted-tet count at three times the oracles' difference."""
    m = box_muscle()
    start = _squashed(m)
    if case == "inverted":
        # mirror the upper fifth of the box through its mid-plane: its tets invert
        z = m.verts[:, 2]
        lo, hi = z.min(), z.max()
        cut = hi - 0.2 * (hi - lo)
        start = m.verts.copy()
        up = z > cut
        start[up, 2] = (2 * cut - z[up]).astype(np.float32)
    _, sim, o32 = _pair(start, 1.0, 2, 0.3)
    o64 = O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS, stopped=m.stopped,
                            repair_alpha=1.0, repair_iters=2, repair_sigma_min=0.3, prec="f64", **KW)
    o64.pos[:] = start
    o64.pprev[:] = start
    inv0 = o64.count_inverted()
    tol = 1e-5 * bbox_diag(m.verts)
    for _ in range(2):
        sim.step()
        o32.step()
        o64.step()
        p = sim.positions_np()
        e = np.abs(p - o64.pos).max(1)
        spr = np.abs(o32.pos - o64.pos).max(1)
        print(f"{case}: |gpu-o64| max {e.max():.3e} p99 {np.percentile(e, 99):.3e}; "
              f"|o32-o64| max {spr.max():.3e} p99 {np.percentile(spr, 99):.3e}")
        assert np.isfinite(p).all()
        assert e.max() <= max(tol, 3.0 * spr.max())
        assert np.percentile(e, 99) <= max(tol, 3.0 * np.percentile(spr, 99))
    n_gpu, n32, n64 = sim.count_inverted(), o32.count_inverted(), o64.count_inverted()
    print(f"{case}: inverted at start {inv0}, after gpu {n_gpu} o32 {n32} o64 {n64}")
    assert abs(n_gpu - n64) <= max(3 * abs(n32 - n64), 0.005 * m.tets.shape[0])
    if case == "inverted":
        assert inv0 > 0 and n64 < inv0


def test_repair_off_is_a_noop():
    m = box_muscle()
    start = _squashed(m)
    _, sim, _ = _pair(start, 0.0, 2, 0.3)
    sim.repair_inverted_tets()
    assert np.array_equal(sim.positions_np(), start)


def test_rebuild_constraints_keeps_state_and_adds_attach():
    """MuscleSim.rebuild_constraints (musclesim.py:289-321): without extras the
    rebuilt sim steps exactly as before; ATTACH rows added as reference-schema
    dicts pull their vertices toward the targets."""
    from rlmusclev2_b200.defs import ConstraintType
    m = box_muscle()
    mk = lambda: MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS,  # noqa: E731
                                           device="cuda:0", stopped=m.stopped, **KW)
    a, b, c = mk(), mk(), mk()
    for s in (a, b, c):
        s.step()
    b.rebuild_constraints()
    np.testing.assert_array_equal(a.positions_np(), b.positions_np())
    free = np.nonzero(m.stopped == 0)[0][:8]
    tgt = m.verts[free] + np.array([0.0, 0.01, 0.0], np.float32)
    rows = [dict(type=int(ConstraintType.ATTACH), pts=[int(v), -1, -1, -1], stiffness=1e6, dampingratio=0.0,
                 restlength=0.0, restvector=[*map(float, t), 1.0]) for v, t in zip(free, tgt)]
    n0 = int(c.c_type.shape[0])
    c.rebuild_constraints(rows)
    # the c_* columns (engine.py:1179-1211) follow the rebuilt table
    assert c.c_type.is_cuda and int(c.c_type.shape[0]) == n0 + len(rows)
    at = (c.c_type == int(ConstraintType.ATTACH)).nonzero().flatten()
    want = {int(v): t for v, t in zip(free, tgt)}
    got_pts = c.c_pts[at, 0].tolist()
    assert sorted(got_pts) == sorted(want)
    np.testing.assert_array_equal(c.c_restvector[at, :3].cpu().numpy(), np.stack([want[v] for v in got_pts]))
    for s in (a, b, c):
        s.step()
    np.testing.assert_array_equal(a.positions_np(), b.positions_np())
    pa, pc = a.positions_np()[free], c.positions_np()[free]
    assert (np.linalg.norm(pc - tgt, axis=1) < np.linalg.norm(pa - tgt, axis=1)).all()


def test_bone_attach_blocks_vs_oracle():
    """An "attach" block (create_attach_constraints, builder.py:347-398): the
    masked vertices attach to their nearest bone point at the rest distance;
    when the bone points move, the targets follow (update_attach_targets,
    musclesim.py:564-578).  Against the FP32 oracle with the same rows."""
    from scipy.spatial import cKDTree
    m = box_muscle()
    z = m.verts[:, 2]
    zr = (z - z.min()) / (z.max() - z.min())
    mask = ((zr > 0.1) & (zr < 0.2)).astype(np.float32)
    bones = (m.verts[mask > 0.5][::3] + np.array([0.0, 0.004, 0.0], np.float32)).astype(np.float32)
    att = dict(type="attach", name="bone_attach", mask_name="attachmask", mask_threshold=0.5, stiffness=1e6,
               dampingratio=0.0)
    sim = MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, bone_targets=bones,
                                    constraint_configs=CONS + [att], device="cuda:0", stopped=m.stopped, **KW)
    sim.geo.attachmask = mask
    sim.build_constraints()
    src = np.nonzero(mask > 0.5)[0]
    d, tgt = cKDTree(bones).query(m.verts[src], k=1)
    assert np.array_equal(np.sort(sim._attach_src), src)
    orc = O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS, stopped=m.stopped,
                            attach=(src, bones[tgt], d, 1e6, 0.0), prec="f32", **KW)
    tol = 1e-5 * bbox_diag(m.verts)
    rows = np.nonzero(orc.c_type == O.T_ATTACH)[0]
    for frame in range(3):
        if frame == 2:  # the bones move: the attach targets follow
            moved = (bones + np.array([0.0, 0.0, 0.005], np.float32)).astype(np.float32)
            sim.bone_pos = moved
            orc.c_rv[rows, :3] = moved[tgt]
        sim.step()
        orc.step()
        err = np.abs(sim.positions_np() - orc.pos).max()
        print(f"bone attach frame {frame}: |gpu-o32| {err:.3e} (tol {tol:.3e})")
        assert err <= tol
    assert np.abs(orc.pos - m.verts).max() > 10 * tol


def test_state_helpers_and_lbs_drive():
    """reset, save_predicted_positions / get_insertion_force, set_lbs_T_rel /
    apply_lbs (musclesim.py:555-656) against their numpy definitions."""
    m = box_muscle()
    sim = MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CONS, device="cuda:0",
                                    stopped=m.stopped, **KW)
    sim.step()
    sim.reset()
    assert np.array_equal(sim.positions_np(), m.verts) and not sim.vel.numpy().any() and sim.step_cnt == 1
    ids = np.arange(0, m.verts.shape[0], 7)
    sim.integrate()
    sim.save_predicted_positions(ids)
    pred = sim.positions_np()[ids].astype(np.float64)
    sim.solve_constraints(run_extras=False)
    sim.apply_dP()
    dts = 1.0 / 240.0
    f = sim.get_insertion_force(ids, dts)
    want = -(sim.mass[ids][:, None] * (sim.positions_np()[ids] - pred) / dts ** 2).sum(0)
    np.testing.assert_allclose(f, want, rtol=1e-5, atol=1e-6)
    # LBS drive: two bones, row-vector transforms q = p R + t
    rng = np.random.default_rng(3)
    Ts = []
    for b in range(2):
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        ang = 0.3 * (b + 1)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        R = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
        Ts.append(np.concatenate([R.reshape(-1), rng.normal(scale=0.01, size=3)]))
    T = np.asarray(Ts, np.float32).reshape(-1)
    vb = rng.integers(-1, 2, size=m.verts.shape[0]).astype(np.int32)
    cur = sim.positions_np().astype(np.float64)
    sim.set_lbs_T_rel(T)
    sim.apply_lbs(vb, blend=0.7)
    got = sim.positions_np()
    want = cur.copy()
    T2 = T.reshape(2, 12).astype(np.float64)
    for b in range(2):
        sel = vb == b
        q = m.verts[sel].astype(np.float64) @ T2[b, :9].reshape(3, 3) + T2[b, 9:]
        want[sel] = (1 - 0.7) * cur[sel] + 0.7 * q
    np.testing.assert_allclose(got, want, atol=2e-6)
