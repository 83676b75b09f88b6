"""Houdini JSON ``.geo`` assets: the reader and per-frame writer the reference's
asset pipeline uses (``util/geo_io.py``), for rest meshes (``restpos.geo``),
pin-target frames (``cons_<frame>.geo``) and headless position export.

A ``.geo`` file is a JSON "pair list" ``[key0, value0, key1, value1, ...]``
(nested pair lists below it).  Point attributes are ``[meta, data]`` pairs;
the payload sits under ``tuples`` (vectors, one row per point) or ``arrays``
(a list holding one array per component; scalar attributes are read as that
one array).  Tetrahedra come from the topology's ``pointref.indices`` with the
count of the ``Tetrahedron_run`` primitive block; point groups are ``ordered``
index lists or ``unordered`` boolean run-length codes.  Reading follows the
reference reader's results field for field (``GeoFile``, geo_io.py:42-209);
writing rewrites ``P`` (and optional ``is_collide`` / ``pen_depth`` point
attributes) in a template and keeps everything else (``GeoWriter``,
geo_io.py:265-309).
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np


def _pairs(lst) -> dict:
    """Pair list -> dict (later duplicates win, as a dict built from zip)."""
    return dict(zip(lst[0::2], lst[1::2]))


def _payload(values_pairs):
    """The numeric payload of an attribute's ``values`` pair list."""
    d = _pairs(values_pairs)
    for key in ("tuples", "arrays", "rawpagedata"):
        if key in d:
            return d[key]
    raise KeyError("attribute values carry neither 'tuples' nor 'arrays'")


def _rle_indices(code) -> np.ndarray:
    """['boolRLE', [count, flag, count, flag, ...]] -> indices of the set runs."""
    if not code or code[0] != "boolRLE":
        return np.zeros(0, np.int32)
    runs = code[1]
    counts = np.asarray(runs[0::2], np.int64)
    flags = np.asarray(runs[1::2], bool)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]]) if counts.size else counts
    idx = [np.arange(s, s + c) for s, c, f in zip(starts, counts, flags) if f]
    return (np.concatenate(idx) if idx else np.zeros(0)).astype(np.int32)


def _squeeze_scalar(a: np.ndarray) -> np.ndarray:
    return a[0] if a.ndim == 2 and a.shape[0] == 1 else a


class GeoFile:
    """Parsed ``.geo``: positions, tet indices, named point / primitive
    attributes and point groups (the reference's GeoFile interface)."""

    def __init__(self, path: str | Path):
        with open(path, "r") as fp:
            root = _pairs(json.load(fp))
        attrs = _pairs(root.get("attributes", []))
        self._attrs: dict[str, np.ndarray] = {}
        self._raw: dict[str, list] = {}  # payloads as stored (the typed accessors read these)
        for meta, data in attrs.get("pointattributes", []):
            name = _pairs(meta)["name"]
            d = _pairs(data)
            if "values" in d:
                self._raw[name] = _payload(d["values"])
                self._attrs[name] = _squeeze_scalar(np.asarray(self._raw[name]))
        self._prim_attrs: dict[str, np.ndarray] = {}
        self._prim_strings: dict[str, list] = {}
        for meta, data in attrs.get("primitiveattributes", []):
            name = _pairs(meta)["name"]
            d = _pairs(data)
            if "strings" in d and "indices" in d:
                arr = _pairs(d["indices"]).get("arrays")
                if arr is not None:
                    self._prim_attrs[name] = np.asarray(arr).ravel().astype(np.int32)
                    self._prim_strings[name] = list(d["strings"])
            elif "values" in d:
                self._prim_attrs[name] = _squeeze_scalar(np.asarray(_payload(d["values"])))
        indices = np.asarray(_pairs(_pairs(root["topology"])["pointref"])["indices"], np.int32)
        n_tets = 0
        for blk in root.get("primitives", []):
            if _pairs(blk[0]).get("type") == "Tetrahedron_run":
                n_tets = int(_pairs(blk[1])["nprimitives"])
                break
        if n_tets > 0:
            self._tets = indices[: 4 * n_tets].reshape(n_tets, 4)
        else:
            npr = int(root.get("primitivecount", 0))
            self._tets = indices.reshape(npr, indices.size // npr) if npr > 0 and indices.size else \
                indices.reshape(0, 0)
        self._groups: dict[str, np.ndarray] = {}
        for meta, body in root.get("pointgroups", []):
            sel = _pairs(_pairs(body)["selection"])
            if "ordered" in sel:
                self._groups[_pairs(meta)["name"]] = np.asarray(sel["ordered"], np.int32)
            elif "unordered" in sel:
                self._groups[_pairs(meta)["name"]] = _rle_indices(sel["unordered"])

    # the reference reader's typed accessors (geo_io.py:151-209)
    @property
    def positions(self) -> np.ndarray:
        if "P" not in self._raw:
            raise KeyError("attribute 'P' not present in this .geo")
        return np.asarray(self._raw["P"], np.float32)

    @property
    def tet_indices(self) -> np.ndarray:
        return self._tets

    @property
    def gluetoanimation(self) -> np.ndarray:
        # absent -> all False, one per point (the reference reader's fallback)
        if "gluetoanimation" in self._raw:
            return np.asarray(self._raw["gluetoanimation"][0], np.bool_)
        n = len(self._raw["P"]) if "P" in self._raw else 0
        return np.zeros(n, np.bool_)

    @property
    def pts(self) -> np.ndarray:
        if "pts" not in self._raw:
            raise KeyError("attribute 'pts' not present in this .geo")
        return np.asarray(self._raw["pts"][0], np.int32)

    @property
    def target_pos(self) -> np.ndarray:
        if "target_pos" not in self._raw:
            raise KeyError("attribute 'target_pos' not present in this .geo")
        return np.asarray(self._raw["target_pos"], np.float32)

    def point_attr(self, name: str) -> np.ndarray:
        if name not in self._attrs:
            raise KeyError(f"point attribute '{name}' not in {sorted(self._attrs)}")
        return self._attrs[name]

    def has_point_attr(self, name: str) -> bool:
        return name in self._attrs

    def has_point_group(self, name: str) -> bool:
        return name in self._groups

    def point_group(self, name: str) -> np.ndarray:
        if name not in self._groups:
            raise KeyError(f"point group '{name}' not in {sorted(self._groups)}")
        return self._groups[name]

    def has_prim_attr(self, name: str) -> bool:
        return name in self._prim_attrs

    def prim_attr(self, name: str) -> np.ndarray:
        if name not in self._prim_attrs:
            raise KeyError(f"prim attribute '{name}' not in {sorted(self._prim_attrs)}")
        return self._prim_attrs[name]

    def prim_attr_strings(self, name: str) -> list:
        return self._prim_strings.get(name, [])


# ------------------------------------------------------------------ writing
def _point_attr(name: str, values: np.ndarray):
    """[meta, data] of a point attribute: fpreal32 / int32 tuples for vectors,
    one array for scalars."""
    a = np.asarray(values)
    integer = np.issubdtype(a.dtype, np.integer) or a.dtype == np.bool_
    storage = "int32" if integer else "fpreal32"
    conv = (lambda x: int(x)) if integer else (lambda x: float(x))
    meta = ["scope", "public", "type", "numeric", "name", name, "options", {}]
    if a.ndim == 1:
        size, vals = 1, ["size", 1, "storage", storage, "arrays", [[conv(x) for x in a]]]
    else:
        size = int(a.shape[1])
        vals = ["size", size, "storage", storage, "tuples", [[conv(x) for x in row] for row in a]]
    data = ["size", size, "storage", storage, "defaults", ["size", 1, "storage", "fpreal64", "values", [0]],
            "values", vals]
    return [meta, data]


def _rle(indices: np.ndarray, n: int) -> list:
    flags = np.zeros(n, bool)
    flags[np.asarray(indices, np.int64)] = True
    runs, i = [], 0
    while i < n:
        j = i
        while j < n and flags[j] == flags[i]:
            j += 1
        runs += [j - i, bool(flags[i])]
        i = j
    return ["boolRLE", runs]


def write_geo(path: str | Path, positions: np.ndarray, tets: np.ndarray | None = None,
              point_attrs: dict | None = None, prim_attrs: dict | None = None,
              prim_string_attrs: dict | None = None, groups: dict | None = None,
              unordered_groups: dict | None = None, tris: np.ndarray | None = None) -> None:
    """Write a ``.geo`` pair list that GeoFile (and the reference's reader)
    parses: ``P`` as fpreal32 tuples, tets as one ``Tetrahedron_run``,
    ``point_attrs`` (name -> (N,) or (N,k)), numeric ``prim_attrs``,
    ``prim_string_attrs`` (name -> (strings, per-tet index)), point groups as
    ordered lists (``groups``) or boolean run-length codes (``unordered_groups``).
    ``tris`` instead of ``tets`` writes a triangle surface (one polygon run, the
    layout of the reference's bone_<frame>.geo files)."""
    pos = np.asarray(positions, np.float32)
    n = int(pos.shape[0])
    if tris is not None and tets is not None:
        raise ValueError("write_geo: tets or tris, not both")
    t = (np.asarray(tris, np.int64).reshape(-1, 3) if tris is not None else
         np.zeros((0, 4), np.int64) if tets is None else np.asarray(tets, np.int64))
    run = "Polygon_run" if tris is not None else "Tetrahedron_run"
    pattrs = [_point_attr("P", pos)] + [_point_attr(k, v) for k, v in (point_attrs or {}).items()]
    prattrs = []
    for k, v in (prim_attrs or {}).items():
        prattrs.append(_point_attr(k, v))
    for k, (strings, idx) in (prim_string_attrs or {}).items():
        meta = ["scope", "public", "type", "string", "name", k, "options", {}]
        data = ["size", 1, "storage", "int32", "strings", list(strings),
                "indices", ["size", 1, "storage", "int32", "arrays", [[int(x) for x in idx]]]]
        prattrs.append([meta, data])
    pgroups = [[["name", k], ["selection", ["ordered", [int(x) for x in v]]]] for k, v in (groups or {}).items()]
    pgroups += [[["name", k], ["selection", ["unordered", _rle(v, n)]]] for k, v in (unordered_groups or {}).items()]
    root = ["fileversion", "19.5", "pointcount", n, "vertexcount", int(t.size), "primitivecount", int(t.shape[0]),
            "topology", ["pointref", ["indices", [int(x) for x in t.reshape(-1)]]],
            "attributes", ["pointattributes", pattrs, "primitiveattributes", prattrs],
            "primitives", [[["type", run], ["startvertex", 0, "nprimitives", int(t.shape[0])]]]
            if t.shape[0] else [],
            "pointgroups", pgroups]
    with open(path, "w") as fp:
        json.dump(root, fp)


class GeoWriter:
    """Per-frame export into a template ``.geo``: each write replaces the
    template's ``P`` and, when given, an int32 ``is_collide`` and an fpreal32
    ``pen_depth`` point attribute (added if the template lacks them); every
    other field is written back unchanged (GeoWriter, geo_io.py:265-309)."""

    def __init__(self, template_path: str | Path):
        with open(template_path, "r") as fp:
            self._root = json.load(fp)
        root = _pairs(self._root)
        self._n = int(root["pointcount"])
        self._pattrs = _pairs(root["attributes"])["pointattributes"]  # live reference into self._root

    def _find(self, name):
        for entry in self._pattrs:
            if _pairs(entry[0]).get("name") == name:
                return entry
        return None

    @staticmethod
    def _set(pairlist, key, value) -> bool:
        for i in range(0, len(pairlist) - 1, 2):
            if pairlist[i] == key:
                pairlist[i + 1] = value
                return True
        return False

    def _scalar(self, name, values, integer: bool):
        a = np.asarray(values, np.int32 if integer else np.float32).reshape(-1)
        if a.shape[0] != self._n:
            raise ValueError(f"{name} has {a.shape[0]} values, the template has {self._n} points")
        entry = self._find(name)
        if entry is None:
            self._pattrs.append(_point_attr(name, a))
        else:
            vals = _pairs(entry[1])["values"]
            self._set(vals, "arrays", [[int(x) if integer else float(x) for x in a]])

    def write(self, out_path: str | Path, positions: np.ndarray, is_collide: np.ndarray | None = None,
              pen_depth: np.ndarray | None = None) -> None:
        pos = np.asarray(positions, np.float32)
        if pos.shape[0] != self._n:
            raise ValueError(f"positions has {pos.shape[0]} points, the template has {self._n}")
        p = self._find("P")
        if p is None:
            raise KeyError("template .geo has no 'P' attribute")
        self._set(_pairs(p[1])["values"], "tuples", pos.tolist())
        if is_collide is not None:
            self._scalar("is_collide", is_collide, True)
        if pen_depth is not None:
            self._scalar("pen_depth", pen_depth, False)
        with open(out_path, "w") as fp:
            json.dump(self._root, fp)


def read_geo_attr(path: str | Path, attr: str) -> np.ndarray:
    """One attribute of a .geo: "P" (float32 positions) or "target_pos"
    (read_geo_attr_cached, geo_io.py:312-333, without the on-disk cache)."""
    g = GeoFile(path)
    return g.positions if attr == "P" else getattr(g, attr)


def read_cons_frame(cons_dir: str | Path, frame: int) -> np.ndarray:
    """``target_pos`` of ``cons_<frame>.geo`` (geo_io.py:336-338)."""
    return GeoFile(Path(cons_dir) / f"cons_{frame}.geo").target_pos


def scene_from_geo(rest_path: str | Path):
    """A Scene from a ``restpos.geo`` asset, as MultiGridSim reads one
    (mg/mg.py:300-350): points and tets, the fiber field ``materialW`` (+x when absent), the
    ``tendonmask`` (0 when absent), the muscle of each tet from the
    ``muscle_id`` primitive attribute (0 when absent), the outward surface from
    the tets.  The asset carries no capsule skeleton: the scene has no bones,
    so the targets come from ``cons_<frame>.geo`` frames (target_mode="points")."""
    from .meshgen import Scene, boundary_faces, orient_faces_outward, orient_tets
    g = GeoFile(rest_path)
    verts = g.positions.astype(np.float32)
    nv = verts.shape[0]
    # every tet positive with the pt3 reference vertex (the reference loader's
    # fix_tet_winding makes them all negative that way; the constraints see the
    # same shapes either way, and the synthetic scenes use this orientation)
    tets = orient_tets(verts, np.asarray(g.tet_indices, np.int64)).astype(np.int32)
    fib = (g.point_attr("materialW").astype(np.float32).reshape(nv, 3) if g.has_point_attr("materialW")
           else np.tile(np.array([1.0, 0.0, 0.0], np.float32), (nv, 1)))
    tendon = (g.point_attr("tendonmask").astype(np.float32).reshape(nv) if g.has_point_attr("tendonmask")
              else np.zeros(nv, np.float32))
    tpart = (g.prim_attr("muscle_id").astype(np.int32).reshape(-1) if g.has_prim_attr("muscle_id")
             else np.zeros(tets.shape[0], np.int32))
    vpart = np.zeros(nv, np.int32)
    vpart[tets.reshape(-1)] = np.repeat(tpart, 4)
    faces, opp = boundary_faces(tets)
    surf = orient_faces_outward(verts, faces, opp).astype(np.int32)
    z3, z1 = np.zeros((0, 3), np.float32), np.zeros(0, np.float32)
    return Scene(verts=verts, tets=tets, tet_part=tpart, vert_part=vpart, v_tendon=tendon, v_fiber=fib,
                 surface_tris=surf, bone_center=z3, bone_axis=z3, bone_half=z1, bone_radius=z1,
                 vert_bone=np.zeros((nv, 2), np.int32), vert_bw=np.zeros(nv, np.float32), traj={}, aniso_muscle=-1,
                 meta=dict(source=str(rest_path), muscle_names=list(g.prim_attr_strings("muscle_id"))))
