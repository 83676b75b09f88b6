"""A rest mesh read from a .geo asset with pin-to-target frames from
cons_<frame>.geo (the reference's default target_mode="points",
mg/mg.py:300-350, 448-458, 1238-1250).  The asset is the synthetic scene
written out (positions, tets, tendonmask, materialW, muscle_id), and its cons
frames carry, bit for bit, the targets the synthetic run with
target_mode="lbs" computes on the device for every vertex; the two runs must
then agree (to the order of the float atomics of the boundary sums)."""
import numpy as np
import pytest

from rlmusclev2_b200.geo import write_geo
from rlmusclev2_b200.meshgen import humanv2_scene
from rlmusclev2_b200.mg import MultiGridSim, load_config

pytestmark = pytest.mark.gpu


def test_geo_asset_with_cons_frames_matches_the_synthetic_run(tmp_path):
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=0, box=(0.35, 0.35, 0.35))
    write_geo(tmp_path / "restpos.geo", sc.verts, sc.tets,
              point_attrs={"tendonmask": sc.v_tendon, "materialW": sc.v_fiber},
              prim_string_attrs={"muscle_id": ([f"m{i}" for i in range(5)], sc.tet_part)})
    base = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    base["demo"]["collision"]["enabled"] = False
    for c in base["constraints"]:
        if c.get("name") == "fiber":
            c["region"] = "all"
    ref_cfg = dict(base, target_mode="lbs")
    ref = MultiGridSim(ref_cfg, scene=sc)
    # cons frames carry the synthetic run's own device targets, bit for bit
    cons = tmp_path / "cons"
    cons.mkdir()
    pts = np.arange(sc.verts.shape[0], dtype=np.int32)
    tg = {}
    for f in range(1, 5):
        ref.load_frame_targets(f)
        ref._targets_kernel()
        ref.synchronize()
        t = np.empty((ref.NV, 3), np.float32)
        t[ref.layout.perm] = ref._pin_tgt[:, :3].cpu().numpy()
        tg[f] = t
        write_geo(cons / f"cons_{f}.geo", t, None, point_attrs={"pts": pts, "target_pos": t})
    geo_cfg = {k: v for k, v in base.items() if k != "synthetic"}
    geo_cfg.update(rest_path=str(tmp_path / "restpos.geo"), cons_dir=str(cons), target_mode="points")
    sim = MultiGridSim(geo_cfg)
    assert sim.NV == ref.NV and sim.NT == ref.NT and sim.scene.n_bones == 0
    assert np.array_equal(sim.pin_active_np, ref.pin_active_np)
    sim.load_frame_targets(3)
    sim._targets_kernel()
    sim.synchronize()
    got = np.empty((sim.NV, 3), np.float32)
    got[sim.layout.perm] = sim._pin_tgt[:, :3].cpu().numpy()
    np.testing.assert_array_equal(got, tg[3])
    for f in range(1, 5):
        a = sc.activation(f)
        for s in (ref, sim):
            s.set_fiber_activation(a)
            s.step_frame(f)
    pr, pg = ref.positions_np(), sim.positions_np()
    err = np.abs(pr - pg).max()
    print(f"geo asset run vs synthetic run: max |diff| {err:.2e} m")
    assert np.isfinite(pg).all()
    assert err < 1e-6


def test_musclesim_from_geo_config_matches_from_procedural(tmp_path):
    """MuscleSim(cfg) (musclesim.py:44-92) on a .geo rest mesh and on a text
    USD TetMesh: the box muscle written out with its per-vertex fiber field
    steps exactly like MuscleSim.from_procedural on the same arrays."""
    from rlmusclev2_b200 import MuscleSim
    from tests._cases import CFG1, CFG1_CONSTRAINTS, cfg1_mesh
    m = cfg1_mesh()
    vf = np.tile(np.array([0.0, 0.0, 1.0], np.float32), (m.verts.shape[0], 1))
    write_geo(tmp_path / "box.geo", m.verts, m.tets, point_attrs={"materialW": vf})
    cfg = dict(geo_path=str(tmp_path / "box.geo"), constraints=CFG1_CONSTRAINTS, dt=CFG1["dts"],
               num_substeps=CFG1["num_substeps"], density=CFG1["density"], veldamping=CFG1["veldamping"],
               gravity=CFG1["gravity"], contraction_ratio=0.0, fiber_stiffness_scale=1.0)
    a = MuscleSim(cfg)
    b = MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                                  device="cuda:0", **CFG1)
    for s in (a, b):
        s.stopped = m.stopped
    for _ in range(2):
        a.step()
        b.step()
    err = float(np.abs(a.positions_np() - b.positions_np()).max())
    print(f"MuscleSim(cfg) from .geo vs from_procedural: max |diff| {err:.2e} m")
    assert err <= 1e-7
    # the same mesh from a text USD layer (util/mesh_io.py:93-150 without pxr)
    from rlmusclev2_b200.usd import write_usda_tetmesh
    write_usda_tetmesh(tmp_path / "box.usda", m.verts, m.tets, {"materialW": vf})
    c = MuscleSim(dict(cfg, geo_path=str(tmp_path / "box.usda")))
    c.stopped = m.stopped
    for _ in range(2):
        c.step()
    err_u = float(np.abs(c.positions_np() - b.positions_np()).max())
    print(f"MuscleSim(cfg) from .usda vs from_procedural: max |diff| {err_u:.2e} m")
    assert err_u <= 1e-7
    with pytest.raises(NotImplementedError, match="rest meshes are read from"):
        MuscleSim(dict(cfg, geo_path=str(tmp_path / "box.obj")))


def test_lbs_target_file_matches_the_device_lbs_run(tmp_path):
    """target_mode="lbs" with lbs_target_npz (mg.py:1176-1214): a sequence
    file holding, bit for bit, the targets the device computes for frames 1-4
    drives the same frames as the device computation; a fractional frame
    blends the two frames around it."""
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=0, box=(0.35, 0.35, 0.35))
    base = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    base["demo"]["collision"]["enabled"] = False
    ref = MultiGridSim(dict(base, target_mode="lbs"), scene=sc)
    frames = np.arange(1, 5, dtype=np.int32)
    pts = np.empty((4, ref.NV, 3), np.float32)
    for i, f in enumerate(frames):
        ref.load_frame_targets(int(f))
        ref._targets_kernel()
        ref.synchronize()
        pts[i][ref.layout.perm] = ref._pin_tgt[:, :3].cpu().numpy()
    np.savez(tmp_path / "lbs.npz", points=pts, frames=frames)
    sim = MultiGridSim(dict(base, target_mode="lbs", lbs_target_npz=str(tmp_path / "lbs.npz")), scene=sc)
    sim.load_frame_targets(2.25)
    sim._targets_kernel()
    sim.synchronize()
    got = np.empty((sim.NV, 3), np.float32)
    got[sim.layout.perm] = sim._pin_tgt[:, :3].cpu().numpy()
    np.testing.assert_array_equal(got, (0.75 * pts[1].astype(np.float64) + 0.25 * pts[2]).astype(np.float32))
    for f in frames:
        a = sc.activation(int(f))
        for s in (ref, sim):
            s.set_fiber_activation(a)
            s.step_frame(int(f))
    err = float(np.abs(ref.positions_np() - sim.positions_np()).max())
    print(f"lbs target file vs device lbs: max |diff| {err:.2e} m")
    assert np.isfinite(sim.positions_np()).all()
    assert err < 1e-6
    with pytest.raises(ValueError, match="lbs_target_npz"):
        np.savez(tmp_path / "bad.npz", points=pts[:, :-1], frames=frames)
        MultiGridSim(dict(base, target_mode="lbs", lbs_target_npz=str(tmp_path / "bad.npz")), scene=sc)
