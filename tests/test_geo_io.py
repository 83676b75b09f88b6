"""Houdini .geo reader and writer (rlmusclev2_b200.geo) against the reference's
own reader: tests/golden/geo_small_ref.npz holds what the reference's GeoFile
(src/muscle/util/geo_io.py) read from the two fixture files
(tests/golden/make_geo_golden.py made all three)."""
from pathlib import Path

import numpy as np
import pytest

from rlmusclev2_b200.geo import GeoFile, GeoWriter, _rle_indices, read_cons_frame, write_geo

G = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def ref():
    return np.load(G / "geo_small_ref.npz")


def test_reader_matches_the_reference_reader(ref):
    g = GeoFile(G / "geo_small.geo")
    np.testing.assert_array_equal(g.positions, ref["positions"])
    assert g.positions.dtype == np.float32
    np.testing.assert_array_equal(g.tet_indices, ref["tets"])
    np.testing.assert_array_equal(g.gluetoanimation, ref["gluetoanimation"])
    np.testing.assert_array_equal(g.point_attr("tendonmask"), ref["tendonmask"])
    np.testing.assert_array_equal(g.point_attr("materialW"), ref["materialW"])
    np.testing.assert_array_equal(g.prim_attr("muscle_id"), ref["muscle_id"])
    assert g.prim_attr_strings("muscle_id") == list(ref["muscle_id_strings"])
    np.testing.assert_array_equal(g.point_group("pinned"), ref["pinned"])
    np.testing.assert_array_equal(g.point_group("surface_points"), ref["surface_points"])
    assert g.has_point_attr("tendonmask") and not g.has_point_attr("pinmask")
    with pytest.raises(KeyError):
        g.pts
    c = GeoFile(G / "geo_cons_small.geo")
    np.testing.assert_array_equal(c.pts, ref["cons_pts"])
    np.testing.assert_array_equal(c.target_pos, ref["cons_target"])


def test_writer_replaces_positions_and_keeps_the_rest(tmp_path):
    w = GeoWriter(G / "geo_small.geo")
    g0 = GeoFile(G / "geo_small.geo")
    new = g0.positions + np.float32(0.01)
    w.write(tmp_path / "frame1.geo", new, is_collide=np.arange(new.shape[0]) % 2,
            pen_depth=np.linspace(0, 1, new.shape[0]))
    g1 = GeoFile(tmp_path / "frame1.geo")
    np.testing.assert_array_equal(g1.positions, new)
    np.testing.assert_array_equal(g1.tet_indices, g0.tet_indices)
    np.testing.assert_array_equal(g1.point_attr("materialW"), g0.point_attr("materialW"))
    np.testing.assert_array_equal(g1.point_attr("is_collide"), np.arange(new.shape[0]) % 2)
    assert np.allclose(g1.point_attr("pen_depth"), np.linspace(0, 1, new.shape[0]))
    w.write(tmp_path / "frame2.geo", g0.positions, is_collide=np.ones(new.shape[0], np.int32))
    g2 = GeoFile(tmp_path / "frame2.geo")  # the attribute is overwritten, not appended twice
    np.testing.assert_array_equal(g2.point_attr("is_collide"), np.ones(new.shape[0], np.int32))
    with pytest.raises(ValueError):
        w.write(tmp_path / "bad.geo", g0.positions[:-1])


def test_run_length_groups_and_cons_frames(tmp_path):
    assert _rle_indices(["boolRLE", [3, False, 2, True, 1, False, 4, True]]).tolist() == [3, 4, 6, 7, 8, 9]
    assert _rle_indices(["boolRLE", []]).size == 0
    assert _rle_indices([]).size == 0
    pos = np.random.default_rng(0).random((12, 3)).astype(np.float32)
    write_geo(tmp_path / "cons_5.geo", pos, None, point_attrs={"pts": np.arange(12), "target_pos": pos},
              unordered_groups={"g": [0, 1, 5, 11]})
    np.testing.assert_array_equal(read_cons_frame(tmp_path, 5), pos)
    assert GeoFile(tmp_path / "cons_5.geo").point_group("g").tolist() == [0, 1, 5, 11]
    assert GeoFile(tmp_path / "cons_5.geo").tet_indices.shape == (0, 0)


def test_scene_from_geo_asset():
    from rlmusclev2_b200.geo import scene_from_geo
    sc = scene_from_geo(G / "geo_small.geo")
    g = GeoFile(G / "geo_small.geo")
    assert sc.verts.shape == g.positions.shape and sc.tets.shape == g.tet_indices.shape
    q = sc.verts[sc.tets].astype(np.float64)
    assert (np.linalg.det(np.stack([q[:, 0] - q[:, 3], q[:, 1] - q[:, 3], q[:, 2] - q[:, 3]], 1)) > 0).all()
    np.testing.assert_array_equal(np.sort(sc.tets, 1), np.sort(g.tet_indices, 1))
    np.testing.assert_array_equal(sc.tet_part, g.prim_attr("muscle_id"))
    np.testing.assert_array_equal(sc.v_tendon, g.point_attr("tendonmask").astype(np.float32))
    assert sc.n_bones == 0 and sc.surface_tris.shape[1] == 3 and sc.surface_tris.shape[0] > 0
