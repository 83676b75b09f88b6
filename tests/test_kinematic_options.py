"""Host side of the soft pins (presubframe_pintotarget, mg_coarse_attach_beta)
on the oracle, CPU only: the blend arithmetic, the coarse attach set, and that
both options change the oracle's frames."""
import numpy as np

from oracle import oracle as O
from rlmusclev2_b200.meshgen import humanv2_scene
from rlmusclev2_b200.mg import load_config

CFG3 = "rlmusclev2_b200/configs/humanv2_synth_mg_dcd.json"


def _cfg(presub=0.0, beta=0.0):
    cfg = load_config(CFG3)
    cfg["demo"]["collision"]["sdf_res"] = 48
    cfg["demo"]["self_collision"]["method"] = "none"
    cfg["presubframe_pintotarget"] = presub
    cfg["mg_coarse_attach_beta"] = beta
    return cfg


def _scene():
    return humanv2_scene(seed=2, n_muscles=3, n_bones=3, target_tets=4000, fascia_tets=800, box=(0.25, 0.25, 0.25))


def test_blend_is_one_fma():
    sc = _scene()
    o = O.OracleMultiGridSim(_cfg(), sc, prec="f32")
    rng = np.random.default_rng(0)
    p = rng.standard_normal((1000, 3)).astype(np.float32)
    t = rng.standard_normal((1000, 3)).astype(np.float32)
    got = o.blend(p, t, 0.3)
    d = (t - p).astype(np.float32)
    want = (p.astype(np.float64) + np.float64(np.float32(0.3)) * d.astype(np.float64)).astype(np.float32)
    assert got.dtype == np.float32 and np.array_equal(got, want)
    assert np.abs(o.blend(p, t, 1.0) - t).max() <= 4.8e-7  # snaps to the rounding of p + (t - p)
    assert np.array_equal(o.blend(p, t, 0.0), p)


def test_coarse_attach_set_is_the_referenced_nodes():
    sc = _scene()
    o = O.OracleMultiGridSim(_cfg(beta=0.3), sc, prec="f32")
    ref = np.zeros(o.mg.nv, bool)
    ref[np.unique(o.mg_t[np.abs(o.mg_w) > 0])] = True
    assert np.array_equal(o.mg_attach, ref)
    assert o.mg_attach.any()


def test_options_change_the_frames():
    sc = _scene()
    runs = {}
    for key in ((0.0, 0.0), (0.5, 0.0), (0.0, 0.3)):
        o = O.OracleMultiGridSim(_cfg(*key), sc, prec="f32")
        for f in (1, 2):
            o.step_frame(f)
        assert np.isfinite(o.pos).all()
        runs[key] = o.pos.copy()
    assert np.abs(runs[(0.5, 0.0)] - runs[(0.0, 0.0)]).max() > 1e-5
    assert np.abs(runs[(0.0, 0.3)] - runs[(0.0, 0.0)]).max() > 1e-6


def test_projection_mode_restarts_from_the_prolonged_target():
    """mg_mode="projection" on the oracle: after one substep's V-cycle the
    embedded vertices sit on the prolonged restricted target."""
    sc = _scene()
    cfg = _cfg()
    cfg["mg_mode"] = "projection"
    o = O.OracleMultiGridSim(cfg, sc, prec="f64")
    o.target, _ = o.targets(2)
    o.mg_target = o.restrict(o.target, o.mg_target)
    o.pos[:] = o.pos + 0.01
    o.vcycle()
    e, w, t = o.mg_emb, o.mg_w, o.mg_t
    want = sum(w[:, k:k + 1] * o.mg_target[t[:, k]] for k in range(4))
    assert np.abs(o.pos[e] - want).max() < 1e-12
    # the restricted target reproduces the bone target on the embedded vertices
    assert np.abs(o.pos[e] - o.target[e]).max() < 5e-3


def test_baked_cage_file_round_trips_and_drives_the_same_frames(tmp_path):
    """coarse_npz_path: a missing file is baked and written, a present one is
    loaded with every array unchanged, and the oracle steps the same frames
    from the file as from the in-memory cage."""
    from rlmusclev2_b200.meshgen import CAGE_NPZ_KEYS, build_cage, cage_for_config, load_cage_npz
    sc = _scene()
    path = tmp_path / "cage" / "coarse_cage"   # no ".npz": the name is kept as given
    cfg = _cfg()
    cage_mem = build_cage(sc, spacing=float(cfg.get("mg_cage_spacing", 0.016)))
    cfg["coarse_npz_path"] = str(path)
    cage_file = cage_for_config(sc, cfg)
    assert path.exists()
    with np.load(path) as d:
        assert set(CAGE_NPZ_KEYS) <= set(d.files)
    for k in CAGE_NPZ_KEYS[:-1]:
        assert np.array_equal(getattr(cage_file, k), getattr(cage_mem, k)), k
    assert cage_file.mg_fine_nv == sc.verts.shape[0] and cage_file.lam == cage_mem.lam
    runs = []
    for c in (_cfg(), cfg):
        o = O.OracleMultiGridSim(c, sc, prec="f32")
        for f in (1, 2):
            o.step_frame(f)
        runs.append(o.pos.copy())
    assert np.array_equal(runs[0], runs[1])
    # a file without "lam" is a reference-baked pinv cage: lam = 0
    ref = tmp_path / "ref.npz"
    np.savez(ref, **{k: (np.int64(cage_mem.mg_fine_nv) if k == "mg_fine_nv" else getattr(cage_mem, k))
                     for k in CAGE_NPZ_KEYS})
    assert load_cage_npz(ref, sc.verts.shape[0]).lam == 0.0


def test_cage_file_is_checked_before_use(tmp_path):
    import pytest
    from rlmusclev2_b200.meshgen import build_cage, load_cage_npz, save_cage_npz
    sc = _scene()
    cage = build_cage(sc)
    nv = sc.verts.shape[0]
    good = tmp_path / "good.npz"
    save_cage_npz(cage, good)
    with pytest.raises(ValueError, match="fine NV"):
        load_cage_npz(good, nv + 1)
    bad = dict(np.load(good))
    bad["blk_matoff"] = bad["blk_matoff"].copy()
    bad["blk_matoff"][-1] = bad["minv_flat"].shape[0]
    np.savez(tmp_path / "bad_blk.npz", **bad)
    with pytest.raises(ValueError, match="block table"):
        load_cage_npz(tmp_path / "bad_blk.npz", nv)
    bad = dict(np.load(good))
    bad["coarse_tet"] = bad["coarse_tet"].copy()
    bad["coarse_tet"][0, 0] = bad["coarse_pos"].shape[0]
    np.savez(tmp_path / "bad_tet.npz", **bad)
    with pytest.raises(ValueError, match="coarse_tet"):
        load_cage_npz(tmp_path / "bad_tet.npz", nv)
    bad = dict(np.load(good))
    del bad["uvw"]
    np.savez(tmp_path / "no_uvw.npz", **bad)
    with pytest.raises(ValueError, match="lacks"):
        load_cage_npz(tmp_path / "no_uvw.npz", nv)


def test_lbs_target_file_frames_clamp_and_blend():
    """_lbs_targets (mg.py:1200-1214): frames before and after the sequence
    clamp to its ends, integer frames are the stored frame, fractional frames
    blend the two around them in FP32."""
    from types import SimpleNamespace
    from rlmusclev2_b200.mg import MultiGridSim
    rng = np.random.default_rng(3)
    pts = rng.standard_normal((3, 50, 3)).astype(np.float32)
    s = SimpleNamespace(_lbs_pts=pts, _lbs_f0=5)
    f = MultiGridSim._lbs_targets
    assert np.array_equal(f(s, 2), pts[0]) and np.array_equal(f(s, 9.5), pts[2])
    assert np.array_equal(f(s, 6), pts[1])
    got = f(s, 5.4)
    w = 5.4 - np.floor(5.4)  # a float64 weight: the blend runs in FP64, rounded once
    assert got.dtype == np.float32
    assert np.array_equal(got, ((1.0 - w) * pts[0].astype(np.float64) + w * pts[1]).astype(np.float32))


def test_coarse_in_fine_embedding_reads_interior_points_exactly():
    """coarse_in_fine_embedding (mg.py:903-938): a point inside the fine mesh
    (a fine tet's centroid) gets its enclosing tet with non-negative weights
    that reproduce it; a point outside extrapolates (a negative weight)."""
    from rlmusclev2_b200.meshgen import coarse_in_fine_embedding
    sc = _scene()
    x = sc.verts.astype(np.float64)
    probe = x[sc.tets[::97]].mean(1)
    far = x.max(0) + 0.05
    t, w = coarse_in_fine_embedding(sc.verts, sc.tets, np.vstack([probe, far[None]]))
    rec = np.einsum("nk,nkd->nd", w.astype(np.float64), x[t])
    assert np.abs(rec - np.vstack([probe, far[None]])).max() < 1e-5
    assert (w[:-1] >= -1e-5).all() and np.allclose(w.sum(1), 1.0, atol=1e-5)
    assert w[-1].min() < 0


def test_restrict_modes_change_the_frames():
    """mg_restrict_mode "galerkin" / "none" and mg_sync_restrict "c2f"
    (mg.py:224-246, 1006-1012) each give different frames from the default
    state restriction on the oracle."""
    sc = _scene()
    runs = {}
    for key in (("direct", "galerkin"), ("galerkin", "galerkin"), ("none", "galerkin"), ("direct", "c2f")):
        cfg = _cfg()
        cfg["mg_restrict_mode"], cfg["mg_sync_restrict"] = key
        o = O.OracleMultiGridSim(cfg, sc, prec="f32")
        for f in (1, 2):
            o.step_frame(f)
        runs[key] = o.pos.copy()
    base = runs[("direct", "galerkin")]
    for key, p in runs.items():
        print(key, np.isfinite(p).all(), np.abs(p - base).max())
        if key != ("direct", "galerkin"):
            assert not np.array_equal(p, base), key


def test_gauss_seidel_options_are_refused():
    """use_jacobi=false / use_colored_gs=true (mg.py:353-354,
    musclesim.py:73-74) select Gauss-Seidel solves, which are not on this
    path: both constructors refuse them before touching a device."""
    import pytest
    from rlmusclev2_b200 import MuscleSim
    from rlmusclev2_b200.mg import MultiGridSim
    for key, val in (("use_jacobi", False), ("use_colored_gs", True)):
        cfg = _cfg()
        cfg[key] = val
        with pytest.raises(NotImplementedError, match="Gauss-Seidel"):
            MultiGridSim(cfg, scene=_scene())
        with pytest.raises(NotImplementedError, match="Gauss-Seidel"):
            MuscleSim({key: val, "geo_path": "unused.geo"})


def test_asset_scale_is_an_fp32_product():
    """asset_scale (util/bone_source.py:60-66): positions times the scale in
    FP32, unchanged at 1."""
    from types import SimpleNamespace
    from rlmusclev2_b200.mg import MultiGridSim
    x = np.random.default_rng(5).standard_normal((40, 3)).astype(np.float32) * 100
    f = MultiGridSim._asset_scaled
    assert np.array_equal(f(SimpleNamespace(asset_scale=1.0), x), x)
    got = f(SimpleNamespace(asset_scale=0.01), x)
    assert got.dtype == np.float32 and np.array_equal(got, x * np.float32(0.01))
