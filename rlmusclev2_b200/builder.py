"""Constraint-table construction (vectorised restatement of the reference's
ConstraintBuilderMixin, src/muscle/constraint/builder.py).

The table is the reference's struct-of-arrays layout (engine.py:1179-1211):
c_type, c_pts[4], c_stiffness, c_compressionstiffness, c_dampingratio,
c_tetid, c_L[3], c_restlength, c_restvector[4], c_restdir[3], sorted by type
with a stable sort so that cons_ranges = {type: (offset, count)} matches
MuscleSim.build_constraints (musclesim.py:365-396).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .defs import ConstraintType

_FIELDS = ("c_type", "c_pts", "c_stiffness", "c_compressionstiffness", "c_dampingratio", "c_tetid", "c_L",
           "c_restlength", "c_restvector", "c_restdir")


@dataclass
class ConstraintTable:
    c_type: np.ndarray
    c_pts: np.ndarray
    c_stiffness: np.ndarray
    c_compressionstiffness: np.ndarray
    c_dampingratio: np.ndarray
    c_tetid: np.ndarray
    c_L: np.ndarray
    c_restlength: np.ndarray
    c_restvector: np.ndarray
    c_restdir: np.ndarray
    cons_ranges: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.c_type.shape[0])

    @staticmethod
    def empty() -> "ConstraintTable":
        return ConstraintTable(np.zeros(0, np.int32), np.zeros((0, 4), np.int32), np.zeros(0, np.float32),
                               np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.int32),
                               np.zeros((0, 3), np.float32), np.zeros(0, np.float32), np.zeros((0, 4), np.float32),
                               np.zeros((0, 3), np.float32))

    @staticmethod
    def concat(parts: list["ConstraintTable"]) -> "ConstraintTable":
        if not parts:
            return ConstraintTable.empty()
        return ConstraintTable(*[np.concatenate([getattr(p, f) for p in parts]) for f in _FIELDS])

    def sorted_by_type(self) -> "ConstraintTable":
        """Stable sort by type tag and rebuild cons_ranges (musclesim.py:365-389)."""
        order = np.argsort(self.c_type, kind="stable")
        t = ConstraintTable(*[getattr(self, f)[order] for f in _FIELDS])
        t.cons_ranges = {}
        if t.n:
            types, starts, counts = np.unique(t.c_type, return_index=True, return_counts=True)
            for ty, s, c in zip(types, starts, counts):
                t.cons_ranges[ConstraintType(int(ty))] = (int(s), int(c))
        return t


def tet_rest_data(pos0: np.ndarray, tets: np.ndarray):
    """(B, V0_signed, valid) per tet with the pt3 reference vertex.

    builder.py:28-43 (_batch_compute_tet_rest_matrices): Dm columns are
    p_k - p_3 of the float32 rest positions; V0 = det(Dm)/6 (signed);
    valid = |det| > 1e-30; B = inv(Dm) for valid tets.  As numpy does for
    the reference's float32 arrays: det and inv evaluated in float64 and
    rounded to float32, then V0 = det / 6 in float32.
    """
    tp = np.asarray(pos0, np.float32)[tets]                 # float32 (NT,4,3)
    cols = (tp[:, :3, :] - tp[:, 3:4, :]).astype(np.float64)  # differences in float32, like the reference
    M = np.transpose(cols, (0, 2, 1))
    det = np.linalg.det(M).astype(np.float32)
    valid = np.abs(det) > 1e-30
    B = np.zeros_like(M)
    if valid.any():
        B[valid] = np.linalg.inv(M[valid])
    return B.astype(np.float32), (det / np.float32(6.0)).astype(np.float32), valid


def lumped_mass(pos0: np.ndarray, tets: np.ndarray, density: float) -> tuple[np.ndarray, np.ndarray]:
    """precompute_rest_kernel (engine.py:199-224): rest_volume = |det Dm|/6,
    mass[v] += rest_volume*density/4 over incident tets."""
    tp = pos0[tets].astype(np.float64)
    cols = tp[:, :3, :] - tp[:, 3:4, :]
    vol = np.abs(np.linalg.det(np.transpose(cols, (0, 2, 1)))) / 6.0
    mass = np.zeros(pos0.shape[0], np.float64)
    np.add.at(mass, tets.reshape(-1), np.repeat(vol * float(density) / 4.0, 4))
    return mass.astype(np.float32), vol.astype(np.float32)


def _tet_rows(ctype, tets, idx, stiffness, damp, restlength, restvector, restdir) -> ConstraintTable:
    n = idx.shape[0]
    return ConstraintTable(
        c_type=np.full(n, int(ctype), np.int32),
        c_pts=tets[idx].astype(np.int32),
        c_stiffness=np.full(n, stiffness, np.float32),
        c_compressionstiffness=np.full(n, -1.0, np.float32),
        c_dampingratio=np.full(n, damp, np.float32),
        c_tetid=idx.astype(np.int32),
        c_L=np.zeros((n, 3), np.float32),
        c_restlength=restlength.astype(np.float32),
        c_restvector=np.tile(np.asarray(restvector, np.float32), (n, 1)),
        c_restdir=np.tile(np.asarray(restdir, np.float32), (n, 1)) if restdir is not None else np.zeros((n, 3),
                                                                                                      np.float32),
    )


def _stiffness(params: dict, default: float) -> float:
    if "compliance" in params:
        c = float(params["compliance"])
        return float("inf") if c == 0.0 else 1.0 / c
    return float(params.get("stiffness", default))


def create_tet_volume_constraint(pos0, tets, params, tet_mask=None) -> ConstraintTable:
    """builder.py:155-177."""
    _, V0, valid = tet_rest_data(pos0, tets)
    sel = valid if tet_mask is None else (valid & tet_mask)
    idx = np.nonzero(sel)[0]
    return _tet_rows(ConstraintType.TETVOLUME, tets, idx, _stiffness(params, 1e10), params.get("dampingratio", 0.0),
                     V0[idx], [0.0, 0.0, 0.0, 0.0], None)


def create_tet_arap_constraints(pos0, tets, params, ctype=ConstraintType.TETARAPSVD, tet_mask=None) -> ConstraintTable:
    """builder.py:583-608 (shared by TETARAPSVD and TETARAPANISO)."""
    if ctype not in (ConstraintType.TETARAPSVD, ConstraintType.TETARAPANISO):
        raise NotImplementedError(f"constraint type {ctype!r} is not on the sm_100a path "
                                  "(supported: tetarapsvd, aniso_arap, volume, snh, attach)")
    _, V0, valid = tet_rest_data(pos0, tets)
    sel = valid if tet_mask is None else (valid & tet_mask)
    idx = np.nonzero(sel)[0]
    return _tet_rows(ctype, tets, idx, _stiffness(params, 1e6), params.get("dampingratio", 0.0), V0[idx],
                     [0.0, 0.0, 0.0, 1.0], None)


def create_tet_snh_constraint(pos0, tets, params, tet_mask=None) -> ConstraintTable:
    """builder.py:310-345: stiffness = mu, restdir[0] = lam."""
    _, V0, valid = tet_rest_data(pos0, tets)
    sel = valid if tet_mask is None else (valid & tet_mask)
    idx = np.nonzero(sel)[0]
    mu = float(params.get("mu", params.get("stiffness", 1000.0)))
    lam = float(params.get("lam", 10000.0))
    return _tet_rows(ConstraintType.TETSNH, tets, idx, mu, params.get("dampingratio", 0.0), V0[idx],
                     [0.0, 0.0, 0.0, 1.0], [lam, 0.0, 0.0])


def create_attach_constraints(src: np.ndarray, target: np.ndarray, restlength, stiffness: float, damp: float,
                              tgt_idx=None, tetid=None) -> ConstraintTable:
    """ATTACH rows, pts = [src, -1, tgt, -1] (builder.py:347-398; belly attach mg.py:700-723)."""
    n = src.shape[0]
    pts = np.full((n, 4), -1, np.int32)
    pts[:, 0] = src
    if tgt_idx is not None:
        pts[:, 2] = tgt_idx
    rv = np.ones((n, 4), np.float32)
    rv[:, :3] = target
    return ConstraintTable(
        c_type=np.full(n, int(ConstraintType.ATTACH), np.int32), c_pts=pts,
        c_stiffness=np.full(n, stiffness, np.float32), c_compressionstiffness=np.full(n, -1.0, np.float32),
        c_dampingratio=np.full(n, damp, np.float32),
        c_tetid=(np.full(n, -1, np.int32) if tetid is None else tetid.astype(np.int32)),
        c_L=np.zeros((n, 3), np.float32), c_restlength=np.broadcast_to(np.asarray(restlength, np.float32), (n,)).copy(),
        c_restvector=rv, c_restdir=np.zeros((n, 3), np.float32))


def constraints_from_dicts(rows: list[dict]) -> ConstraintTable:
    """A table from constraint dicts in the reference's schema (builder.py:164-175:
    type, pts[4], stiffness, dampingratio, compressionstiffness, tetid, L[3],
    restlength, restvector[4], restdir[3]); missing keys take the builder's
    defaults (pts -1, compressionstiffness -1, tetid -1, restvector (0, 0, 0, 1))."""
    n = len(rows)
    t = ConstraintTable(
        c_type=np.zeros(n, np.int32), c_pts=np.full((n, 4), -1, np.int32), c_stiffness=np.zeros(n, np.float32),
        c_compressionstiffness=np.full(n, -1.0, np.float32), c_dampingratio=np.zeros(n, np.float32),
        c_tetid=np.full(n, -1, np.int32), c_L=np.zeros((n, 3), np.float32), c_restlength=np.zeros(n, np.float32),
        c_restvector=np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1)), c_restdir=np.zeros((n, 3), np.float32))
    for i, c in enumerate(rows):
        t.c_type[i] = int(c["type"])
        pts = list(c.get("pts", []))[:4]
        t.c_pts[i, :len(pts)] = pts
        t.c_stiffness[i] = float(c.get("stiffness", 0.0))
        t.c_compressionstiffness[i] = float(c.get("compressionstiffness", -1.0))
        t.c_dampingratio[i] = float(c.get("dampingratio", 0.0))
        t.c_tetid[i] = int(c.get("tetid", -1))
        if c.get("L") is not None:
            t.c_L[i] = np.asarray(c["L"], np.float32)[:3]
        t.c_restlength[i] = float(c.get("restlength", 0.0))
        if c.get("restvector") is not None:
            rv = np.asarray(c["restvector"], np.float32).reshape(-1)
            t.c_restvector[i, :rv.shape[0]] = rv[:4]
        if c.get("restdir") is not None:
            t.c_restdir[i] = np.asarray(c["restdir"], np.float32)[:3]
    return t


def collect_raw_constraints(pos0, tets, constraint_configs, tet_masks: dict | None = None) -> ConstraintTable:
    """_collect_raw_constraints (builder.py:610-656) for the tet types of the
    sm_100a path.  ``tet_masks`` optionally restricts a named config to a tet
    subset (e.g. aniso_arap on one muscle, SNH on fascia tets)."""
    parts = []
    tet_masks = tet_masks or {}
    for params in constraint_configs:
        if not params.get("enable", True):
            continue
        ctype = str(params["type"]).lower()
        mask = tet_masks.get(params.get("name", ctype))
        if ctype == "volume":
            parts.append(create_tet_volume_constraint(pos0, tets, params, mask))
        elif ctype == "tetarapsvd":
            parts.append(create_tet_arap_constraints(pos0, tets, params, ConstraintType.TETARAPSVD, mask))
        elif ctype == "aniso_arap":
            parts.append(create_tet_arap_constraints(pos0, tets, params, ConstraintType.TETARAPANISO, mask))
        elif ctype == "snh":
            parts.append(create_tet_snh_constraint(pos0, tets, params, mask))
        elif ctype in ("attach", "pin", "pintotarget", "glue"):
            continue  # vertex constraints are built by the sim from its bone targets
        else:
            raise NotImplementedError(f"constraint type {ctype!r} is not on the sm_100a path "
                                      "(supported: tetarapsvd, aniso_arap, volume, snh, attach)")
    return ConstraintTable.concat(parts)
