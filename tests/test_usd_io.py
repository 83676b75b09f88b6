"""Text USD (.usda) TetMesh reader: the slice of the reference's
_load_mesh_usd (util/mesh_io.py:93-150) that builds a rest mesh -- the first
TetMesh prim (or the one at prim_path), points and tetVertexIndices as
stored, the materialW / tendonmask primvars and every vertex primvar."""
import numpy as np
import pytest

from rlmusclev2_b200.geo import scene_from_geo, write_geo
from rlmusclev2_b200.usd import load_tetmesh_usda, read_usda, scene_from_usda, write_usda_tetmesh
from tests._cases import random_tet_mesh

HANDWRITTEN = '''#usda 1.0
(
    defaultPrim = "character"
    upAxis = "Z"
)

def Xform "character" (
    kind = "component"
)
{
    # a bone surface first: not a TetMesh
    def Mesh "bone"
    {
        int[] faceVertexCounts = [3]
        int[] faceVertexIndices = [0, 1, 2]
        point3f[] points = [(0, 0, 0), (1, 0, 0), (0, 1, 0)]
    }
    def TetMesh "muscle"
    {
        uniform token[] xformOpOrder = ["xformOp:translate"]
        double3 xformOp:translate = (0, 0, 0)
        point3f[] points = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1),
                            (1, 1, 1e-1)]
        int4[] tetVertexIndices = [(0, 1, 2, 3), (1, 2, 3, 4)]
        float3[] primvars:materialW = [(1, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (0.5, 0.5, 0)] (
            interpolation = "vertex"
        )
        float[] primvars:tendonmask = [0, 0.25, 0.5, 0.75, 1] (
            interpolation = "vertex"
        )
        float[] primvars:stiffness = [3, 4] (
            interpolation = "uniform"
        )
        color3f[] primvars:displayColor = [(0.8, 0.2, 0.2)]
    }
    def TetMesh "second"
    {
        point3f[] points = [(0, 0, 0), (2, 0, 0), (0, 2, 0), (0, 0, 2)]
        int4[] tetVertexIndices = [(0, 1, 2, 3)]
    }
}
'''


def test_handwritten_layer(tmp_path):
    p = tmp_path / "m.usda"
    p.write_text(HANDWRITTEN)
    prims = read_usda(p)
    assert [x.path for x in prims] == ["/character", "/character/bone", "/character/muscle", "/character/second"]
    pos, tets, fib, ten, pv = load_tetmesh_usda(p)
    np.testing.assert_array_equal(pos, np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0.1]], np.float32))
    np.testing.assert_array_equal(tets, np.array([[0, 1, 2, 3], [1, 2, 3, 4]], np.int32))
    assert fib.shape == (5, 3) and fib[4, 1] == np.float32(0.5)
    np.testing.assert_array_equal(ten, np.array([0, 0.25, 0.5, 0.75, 1], np.float32))
    assert set(pv) == {"materialW", "tendonmask"}  # only vertex-interpolated primvars
    pos2, tets2, fib2, ten2, _ = load_tetmesh_usda(p, "/character/second")
    assert pos2.shape == (4, 3) and tets2.shape == (1, 4) and fib2 is None and ten2 is None
    with pytest.raises(ValueError, match="not a TetMesh"):
        load_tetmesh_usda(p, "/character/bone")


def test_binary_crate_rejected(tmp_path):
    p = tmp_path / "b.usd"
    p.write_bytes(b"PXR-USDC" + b"\0" * 64)
    with pytest.raises(NotImplementedError, match="binary USD crate"):
        read_usda(p)


def test_written_layer_round_trip_matches_geo_scene(tmp_path):
    verts, tets = random_tet_mesh(n_cube=3)
    rng = np.random.default_rng(3)
    fib = rng.normal(size=verts.shape).astype(np.float32)
    ten = rng.uniform(size=verts.shape[0]).astype(np.float32)
    write_usda_tetmesh(tmp_path / "m.usda", verts, tets, {"materialW": fib, "tendonmask": ten})
    pos, t, f, m, _ = load_tetmesh_usda(tmp_path / "m.usda")
    np.testing.assert_array_equal(pos, verts.astype(np.float32))
    np.testing.assert_array_equal(t, tets.astype(np.int32))
    np.testing.assert_array_equal(f, fib)
    np.testing.assert_array_equal(m, ten)
    write_geo(tmp_path / "m.geo", verts, tets, point_attrs={"materialW": fib, "tendonmask": ten})
    a, b = scene_from_usda(tmp_path / "m.usda"), scene_from_geo(tmp_path / "m.geo")
    for k in ("verts", "tets", "v_fiber", "v_tendon", "surface_tris"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k))
