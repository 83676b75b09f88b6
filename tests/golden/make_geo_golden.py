"""Writes the .geo golden fixture: a small tet mesh with the attributes the
reference's asset pipeline reads (P, tendonmask, materialW, gluetoanimation,
pts, target_pos, a string muscle_id primitive attribute, an ordered and a
run-length-coded point group), written by rlmusclev2_b200.geo.write_geo, then
parsed by the reference's own reader (src/muscle/util/geo_io.py GeoFile); its
results go to geo_small_ref.npz.  Run from the repository root in a container
that has the reference checkout:

    python tests/golden/make_geo_golden.py <reference checkout>
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from rlmusclev2_b200.geo import write_geo  # noqa: E402
from rlmusclev2_b200.meshgen import box_muscle  # noqa: E402


def main(ref_root: str) -> None:
    m = box_muscle(nx=3, ny=3, nz=5, seed=4)
    n = m.verts.shape[0]
    rng = np.random.default_rng(7)
    tendon = np.clip(rng.random(n), 0, 1).astype(np.float32)
    fib = rng.normal(size=(n, 3)).astype(np.float32)
    glue = (rng.random(n) < 0.3).astype(np.int32)
    pts = np.sort(rng.choice(n, 17, replace=False)).astype(np.int32)
    tgt = (m.verts[pts] + rng.normal(scale=1e-3, size=(17, 3))).astype(np.float32)
    strings = ["bicep", "tricep", "deltoid"]
    mid = rng.integers(0, 3, m.tets.shape[0])
    surf = np.unique(m.surface_tris) if hasattr(m, "surface_tris") else np.arange(0, n, 3)
    geo = HERE / "geo_small.geo"
    write_geo(geo, m.verts, m.tets,
              point_attrs={"tendonmask": tendon, "materialW": fib, "gluetoanimation": glue},
              prim_string_attrs={"muscle_id": (strings, mid)},
              groups={"pinned": pts}, unordered_groups={"surface_points": surf})
    # cons frame: pts + target_pos on the same point count (as cons_<frame>.geo carries them)
    cons = HERE / "geo_cons_small.geo"
    write_geo(cons, tgt, None, point_attrs={"pts": pts, "target_pos": tgt})
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from muscle.util.geo_io import GeoFile as RefGeo  # the reference reader
    r, c = RefGeo(str(geo)), RefGeo(str(cons))
    np.savez(HERE / "geo_small_ref.npz", positions=r.positions, tets=r.tet_indices,
             gluetoanimation=r.gluetoanimation, tendonmask=r.point_attr("tendonmask"),
             materialW=r.point_attr("materialW"), muscle_id=r.prim_attr("muscle_id"),
             muscle_id_strings=np.array(r.prim_attr_strings("muscle_id")),
             pinned=r.point_group("pinned"), surface_points=r.point_group("surface_points"),
             cons_pts=c.pts, cons_target=c.target_pos)
    print("wrote", geo, cons, HERE / "geo_small_ref.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
