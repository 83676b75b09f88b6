"""GPU parity of the sm_100a substep against the CPU oracle (through the C ABI).

Tolerances (the project's parity contract): after 10 substeps every vertex
lies within 1e-5 x bounding-box diagonal of the FP32 oracle; the max ARAP
residual matches to 1e-4 relative and the relative volume drift to 1e-4
absolute.  The FP64 oracle's distance is reported alongside.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rlmusclev2_b200 import MuscleSim, XpbdSolver
from rlmusclev2_b200.builder import ConstraintTable, collect_raw_constraints, create_attach_constraints, lumped_mass
from tests._cases import CFG1, CFG1_CONSTRAINTS, bbox_diag, cfg1_mesh, random_tet_mesh

pytestmark = pytest.mark.gpu


def _cfg1_pair(relax, prec_list=("f32", "f64"), **kw):
    m = cfg1_mesh()
    sim = MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                                    device="cuda:0", stopped=m.stopped, relaxation=relax, **CFG1, **kw)
    orcs = {p: O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                                 stopped=m.stopped, relaxation=relax, prec=p, **CFG1) for p in prec_list}
    return m, sim, orcs


@pytest.mark.parametrize("relax", [1.0, 0.25])
def test_cfg1_fused_graph_matches_oracle_after_10_substeps(relax):
    m, sim, orcs = _cfg1_pair(relax)
    sim.step()
    for o in orcs.values():
        o.step()
    p = sim.positions_np()
    tol = 1e-5 * bbox_diag(m.verts)
    err32 = np.abs(p - orcs["f32"].pos).max()
    err64 = np.abs(p - orcs["f64"].pos).max()
    print(f"relax={relax}: max|gpu-oracle32|={err32:.3e} max|gpu-oracle64|={err64:.3e} tol={tol:.3e}")
    assert err32 <= tol and err64 <= tol
    # residual and volume drift
    mt = sim.metrics()
    r_or = orcs["f64"].arap_residual()
    assert abs(mt["resid_max"] - r_or.max()) <= 1e-4 * r_or.max()
    tot = orcs["f32"].total_rest_volume
    drift_gpu = (mt["vol_sum"] - sim.total_rest_volume) / sim.total_rest_volume
    drift_or = (orcs["f64"].total_volume() - tot) / tot
    assert abs(drift_gpu - drift_or) <= 1e-4
    assert mt["n_nonfinite"] == 0 and mt["n_inverted"] == orcs["f32"].count_inverted()


def test_cfg1_eager_program_matches_fused():
    m, sim, orcs = _cfg1_pair(1.0, prec_list=("f32",))
    m2, sim2, _ = _cfg1_pair(1.0, prec_list=())
    sim.step()
    sim2.step_eager()
    orcs["f32"].step()
    tol = 1e-5 * bbox_diag(m.verts)
    assert np.abs(sim2.positions_np() - orcs["f32"].pos).max() <= tol
    assert np.abs(sim2.positions_np() - sim.positions_np()).max() <= tol
    np.testing.assert_allclose(sim2.vel.numpy(), orcs["f32"].vel, atol=tol * 24 * 10 * 4)


def test_cfg1_two_frames_and_graph_replay():
    m, sim, orcs = _cfg1_pair(1.0, prec_list=("f32",))
    tol = 1e-5 * bbox_diag(m.verts)
    for _ in range(2):
        sim.step()
        orcs["f32"].step()
        assert np.abs(sim.positions_np() - orcs["f32"].pos).max() <= tol


def _mixed_problem(seed=3):
    verts, tets = random_tet_mesh(n_cube=4, seed=seed)
    rng = np.random.default_rng(seed)
    nt, nv = tets.shape[0], verts.shape[0]
    snh_mask = np.zeros(nt, bool)
    snh_mask[: nt // 3] = True
    aniso_mask = np.zeros(nt, bool)
    aniso_mask[nt // 4: 3 * nt // 4] = True
    cfgs = [{"type": "tetarapsvd", "name": "arap", "stiffness": 1e6},
            {"type": "volume", "name": "volume", "stiffness": 1e7, "dampingratio": 0.05},
            {"type": "aniso_arap", "name": "fiber", "stiffness": 5e5},
            {"type": "snh", "name": "snh", "mu": 2e4, "lam": 1e6, "dampingratio": 0.1}]
    masks = {"snh": snh_mask, "fiber": aniso_mask, "arap": ~snh_mask}
    table = collect_raw_constraints(verts, tets, cfgs, tet_masks=masks)
    src = np.arange(0, nv, 7)
    tgt = verts[src] + rng.normal(scale=0.002, size=(src.shape[0], 3)).astype(np.float32)
    att = create_attach_constraints(src, tgt, 0.0, 3e5, 0.1)
    table = ConstraintTable.concat([table, att]).sorted_by_type()
    mass, rv = lumped_mass(verts, tets, 1060.0)
    vf = rng.normal(size=(nv, 3)).astype(np.float32)
    vf /= np.linalg.norm(vf, axis=1, keepdims=True)
    act = rng.uniform(0, 1, nt).astype(np.float32)
    tendon = rng.uniform(0, 1, nt).astype(np.float32) * (rng.random(nt) < 0.3)
    deformed = verts + rng.normal(scale=0.0008, size=verts.shape).astype(np.float32)
    prev = verts + rng.normal(scale=0.0004, size=verts.shape).astype(np.float32)
    return verts, tets, table, mass, vf, act, tendon, deformed, prev


def _oracle_table(table):
    return O.Table.from_arrays(table.c_type, table.c_pts, table.c_stiffness, table.c_dampingratio, table.c_tetid,
                               table.c_restlength, table.c_restvector, table.c_restdir)


@pytest.mark.parametrize("fused", [False, True])
def test_mixed_constraints_one_iteration(fused):
    verts, tets, table, mass, vf, act, tendon, deformed, prev = _mixed_problem()
    dt = 1.0 / 240.0
    kw = dict(dt=dt, contraction_ratio=0.4, fiber_stiffness_scale=3.0)
    sim = XpbdSolver(verts, tets, table, mass=mass, v_fiber=vf, tet_tendonmask=tendon, device="cuda:0",
                     tile_tets=64, **kw)
    sim.set_activation(act)
    sim.set_positions(prev, also_prev=True)
    sim.set_positions(deformed)
    _, B, _, _ = O.precompute_rest(verts, tets, 1060.0, "f32")
    res = {}
    for p in ("f32", "f64"):
        o = O.OracleSolver(verts, tets, _oracle_table(table), mass, np.zeros(len(verts), np.int32), B,
                           gravity_vec=(0, 0, 0), v_fiber=vf, activation=act, tendonmask=tendon, prec=p, **kw)
        o.pos[:] = deformed
        o.pprev[:] = prev
        o.project()
        o.apply_dP()
        res[p] = o.pos.copy()
    if fused:
        sim.iterate_fused()
    else:
        sim.project_once()
    got = sim.positions_np()
    moved = np.abs(res["f64"] - deformed).max()
    tol = 1e-5 * bbox_diag(verts)
    e32 = np.abs(got - res["f32"]).max()
    print(f"fused={fused} moved={moved:.3e} err32={e32:.3e} err64={np.abs(got - res['f64']).max():.3e} tol={tol:.3e}")
    assert moved > 10 * tol
    assert e32 <= tol
