"""USD TetMesh rest meshes from text (.usda) layers, without pxr.

The reference reads muscle rest meshes through pxr (util/mesh_io.py:93-150,
``_load_mesh_usd``): the first ``TetMesh`` prim of the stage (or the one at
``prim_path``), its ``points`` and ``tetVertexIndices`` as they are stored
(no transform), and the ``materialW`` (fiber direction) and ``tendonmask``
primvars; every vertex-interpolated primvar is also exposed by name.  pxr is
not installed here, so this module parses the ASCII form of a USD layer
(``#usda 1.0``): ``def``/``over`` prim blocks with their nesting (prim
paths), array-valued attributes (``point3f[]``, ``int4[]``, ``int[]``,
``float[]``, ``float3[]`` ...) and the ``interpolation`` metadata of
primvars.  Binary crate files (.usdc, and .usd files holding one) are
rejected with a clear error; composition arcs (references, payloads,
variants) are not followed.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_NUM = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?|[-+]?inf|nan")
_DEF = re.compile(r'\b(def|over|class)\s+(?:(\w+)\s+)?"([^"]+)"')
_ATTR = re.compile(r"((?:uniform\s+|custom\s+)*)([A-Za-z_]\w*(?:\[\])?)\s+([A-Za-z_][\w:]*)\s*=\s*")


@dataclass
class UsdaPrim:
    path: str
    type_name: str
    attrs: dict = field(default_factory=dict)  # name -> (type, np.ndarray | str, metadata dict)


def _match_close(text: str, i: int, open_ch: str, close_ch: str) -> int:
    """Index just past the bracket that closes text[i] (== open_ch); strings skipped."""
    depth = 0
    n = len(text)
    while i < n:
        c = text[i]
        if c == '"':
            j = text.index('"', i + 1)
            i = j + 1
            continue
        if c == open_ch:
            depth += 1
        elif c == close_ch:
            depth -= 1
            if depth == 0:
                return i + 1
        i += 1
    raise ValueError(f"unbalanced {open_ch}{close_ch} in USDA text")


def _strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        # '#' starts a comment outside strings (the header line is one too)
        q = False
        for k, c in enumerate(line):
            if c == '"':
                q = not q
            elif c == "#" and not q:
                line = line[:k]
                break
        out.append(line)
    return "\n".join(out)


def _parse_block(body: str, path: str, prims: list) -> None:
    """Attributes and child prims of one prim body (the text inside its braces)."""
    i = 0
    n = len(body)
    this = prims[-1] if prims and prims[-1].path == path else None
    while i < n:
        m_def = _DEF.search(body, i)
        m_attr = _ATTR.search(body, i)
        nxt = min([m.start() for m in (m_def, m_attr) if m is not None], default=n)
        if nxt >= n:
            break
        if m_def is not None and m_def.start() == nxt:
            name = m_def.group(3)
            j = m_def.end()
            if j < n and body[j:].lstrip().startswith("("):  # prim metadata
                k = j + (len(body[j:]) - len(body[j:].lstrip()))
                j = _match_close(body, k, "(", ")")
            k = body.index("{", j)
            end = _match_close(body, k, "{", "}")
            child = f"{path.rstrip('/')}/{name}"
            prims.append(UsdaPrim(child, m_def.group(2) or ""))
            _parse_block(body[k + 1:end - 1], child, prims)
            i = end
            continue
        # attribute: value is an array, a parenthesised tuple or a scalar token
        typ, name = m_attr.group(2), m_attr.group(3)
        j = m_attr.end()
        if j < n and body[j] == "[":
            end = _match_close(body, j, "[", "]")
        elif j < n and body[j] == "(":
            end = _match_close(body, j, "(", ")")
        else:
            e = re.compile(r"[\n;]").search(body, j)
            end = e.start() if e else n
        raw = body[j:end]
        meta = {}
        rest = body[end:]
        ws = len(rest) - len(rest.lstrip(" \t"))
        if rest[ws:ws + 1] == "(":
            mend = _match_close(body, end + ws, "(", ")")
            for mk, mv in re.findall(r'(\w+)\s*=\s*"([^"]*)"', body[end + ws:mend]):
                meta[mk] = mv
            end = mend
        if this is not None:
            if typ.startswith(("string", "token", "asset")):
                val = raw.strip()
            else:
                val = np.array([float(x) for x in _NUM.findall(raw)], np.float64)
            this.attrs[name] = (typ, val, meta)
        i = end


def read_usda(path: str | Path) -> list[UsdaPrim]:
    """All prims of a text USD layer, in file order, with their array attributes."""
    path = Path(path)
    data = path.read_bytes()
    if data[:8] == b"PXR-USDC":
        raise NotImplementedError(f"{path.name} is a binary USD crate file; only text (.usda) layers are read "
                                  "(pxr is not installed)")
    text = data.decode("utf-8")
    if not text.lstrip().startswith("#usda"):
        raise ValueError(f"{path.name}: not a text USD layer (no '#usda' header)")
    prims: list[UsdaPrim] = []
    _parse_block(_strip_comments(text), "/", prims)
    return prims


_COMPONENTS = {"point3f": 3, "float3": 3, "normal3f": 3, "vector3f": 3, "color3f": 3, "double3": 3,
               "int4": 4, "int3": 3, "int2": 2, "float2": 2, "texCoord2f": 2}


def _as_array(typ: str, val: np.ndarray) -> np.ndarray:
    base = typ.rstrip("[]")
    k = _COMPONENTS.get(base, 1)
    out = val.reshape(-1, k) if k > 1 else val.reshape(-1)
    return out.astype(np.int32) if base.startswith("int") else out.astype(np.float32)


def load_tetmesh_usda(path: str | Path, prim_path: str | None = None):
    """_load_mesh_usd (util/mesh_io.py:93-150) for a text layer: returns
    (positions, tets, fibers, tendon_mask, primvars) -- positions and tets as
    stored, fibers/tendon_mask from the ``materialW`` / ``tendonmask`` primvars
    (None when absent), primvars every vertex-interpolated primvar by name."""
    prims = read_usda(path)
    tet = None
    for p in prims:
        if (prim_path is None and p.type_name == "TetMesh") or (prim_path is not None and p.path == prim_path):
            tet = p
            break
    if tet is None:
        raise ValueError(f"no TetMesh prim{' ' + prim_path if prim_path else ''} found in {Path(path).name}")
    if tet.type_name != "TetMesh":
        raise ValueError(f"prim {tet.path} is a {tet.type_name or 'typeless prim'}, not a TetMesh")
    if "points" not in tet.attrs or "tetVertexIndices" not in tet.attrs:
        raise ValueError(f"TetMesh {tet.path} lacks points or tetVertexIndices")
    pos = _as_array(*tet.attrs["points"][:2]).reshape(-1, 3)
    tets = _as_array(*tet.attrs["tetVertexIndices"][:2]).reshape(-1, 4)
    primvars = {}
    for name, (typ, val, meta) in tet.attrs.items():
        if name.startswith("primvars:") and not isinstance(val, str) and meta.get("interpolation") == "vertex":
            primvars[name[len("primvars:"):]] = _as_array(typ, val)
    fib = primvars.get("materialW")
    ten = primvars.get("tendonmask")
    return pos, tets, fib, ten, primvars


def write_usda_tetmesh(path: str | Path, positions: np.ndarray, tets: np.ndarray, primvars: dict | None = None,
                       prim_path: str = "/character/muscle") -> None:
    """A text layer holding one TetMesh (points, tetVertexIndices and
    vertex-interpolated primvars: float for (N,), float3 for (N,3))."""
    parts = [p for p in prim_path.strip("/").split("/") if p]
    lines = ["#usda 1.0", ""]
    ind = ""
    for k, name in enumerate(parts):
        typ = "TetMesh" if k == len(parts) - 1 else "Xform"
        lines += [f'{ind}def {typ} "{name}"', f"{ind}{{"]
        ind += "    "
    fmt = lambda a: ", ".join("(" + ", ".join(repr(float(x)) for x in r) + ")" for r in a)  # noqa: E731
    lines.append(f"{ind}point3f[] points = [{fmt(np.asarray(positions, np.float32))}]")
    tt = np.asarray(tets, np.int64)
    lines.append(f"{ind}int4[] tetVertexIndices = [" + ", ".join("(" + ", ".join(str(int(x)) for x in r) + ")"
                                                            for r in tt) + "]")
    for name, arr in (primvars or {}).items():
        a = np.asarray(arr, np.float32)
        if a.ndim == 1:
            body = ", ".join(repr(float(x)) for x in a)
            lines.append(f"{ind}float[] primvars:{name} = [{body}] (")
        else:
            lines.append(f"{ind}float3[] primvars:{name} = [{fmt(a)}] (")
        lines += [f'{ind}    interpolation = "vertex"', f"{ind})"]
    for _ in parts:
        ind = ind[:-4]
        lines.append(f"{ind}}}")
    Path(path).write_text("\n".join(lines) + "\n")


def scene_from_usda(path: str | Path, prim_path: str | None = None):
    """A rest Scene from a text USD TetMesh, as geo.scene_from_geo builds one
    from a .geo asset: points, positively oriented tets, ``materialW`` (+x when
    absent), ``tendonmask`` (0 when absent), one part, the outward surface; no
    bones (targets then come from cons frames)."""
    from .meshgen import Scene, boundary_faces, orient_faces_outward, orient_tets
    pos, tets, fib, ten, _ = load_tetmesh_usda(path, prim_path)
    verts = pos.astype(np.float32)
    nv = verts.shape[0]
    tets = orient_tets(verts, tets.astype(np.int64)).astype(np.int32)
    fib = fib.reshape(nv, 3) if fib is not None else np.tile(np.array([1.0, 0.0, 0.0], np.float32), (nv, 1))
    ten = ten.reshape(nv) if ten is not None else np.zeros(nv, np.float32)
    faces, opp = boundary_faces(tets)
    surf = orient_faces_outward(verts, faces, opp).astype(np.int32)
    z3, z1 = np.zeros((0, 3), np.float32), np.zeros(0, np.float32)
    return Scene(verts=verts, tets=tets, tet_part=np.zeros(tets.shape[0], np.int32), vert_part=np.zeros(nv, np.int32),
                 v_tendon=ten.astype(np.float32), v_fiber=fib.astype(np.float32), surface_tris=surf, bone_center=z3,
                 bone_axis=z3, bone_half=z1, bone_radius=z1, vert_bone=np.zeros((nv, 2), np.int32),
                 vert_bw=np.zeros(nv, np.float32), traj={}, aniso_muscle=-1, meta=dict(source=str(path)))
