"""Device layout: Morton tiles of tets, tile-grouped vertex order, packed tet
streams and the material table (host-side setup, run once per mesh).

Layout in HBM (library order, see include/xpbd_b200.h):

* tets are sorted by the Morton code of their rest centroid and cut into
  tiles of ``tile_tets`` consecutive tets (one CTA each);
* vertices are renumbered so that each tile's interior vertices (touched by
  that tile only) are contiguous, followed by the boundary vertices first seen
  in that tile; within those groups vertices keep Morton order;
* per tet 52 bytes in four coalesced streams: tet_q (16-bit tile-local vertex
  indices, material id, V0), tet_b0/tet_b1 (B rows 0-1 and B10..B21), tet_b2.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from .builder import ConstraintTable, tet_rest_data
from .defs import ConstraintType


def morton_codes(x: np.ndarray, lo: np.ndarray, hi: np.ndarray, bits: int = 10) -> np.ndarray:
    """30-bit 3D Morton codes of points x quantised over the box [lo, hi]."""
    ext = np.maximum(hi - lo, 1e-30)
    q = np.clip(((x - lo) / ext * ((1 << bits) - 1)).astype(np.int64), 0, (1 << bits) - 1).astype(np.uint64)

    def spread(v):
        v = v & np.uint64(0x3FF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x09249249)
        return v

    return spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)) | (spread(q[:, 2]) << np.uint64(2))


@dataclass
class TileLayout:
    n_verts: int
    n_tets: int
    perm: np.ndarray          # new vertex id -> user vertex id
    inv: np.ndarray           # user vertex id -> new vertex id
    tet_perm: np.ndarray      # new tet id -> user tet id
    tet_inv: np.ndarray       # user tet id -> new tet id
    tets_new: np.ndarray      # (NT,4) tets in new order with new vertex ids
    tile_vptr: np.ndarray
    tile_nint: np.ndarray
    tile_tptr: np.ndarray
    tile_verts: np.ndarray
    bnd_verts: np.ndarray
    max_tile_verts: int
    tet_q: np.ndarray         # (NT,4) uint32
    tet_b0: np.ndarray        # (NT,4) float32
    tet_b1: np.ndarray        # (NT,4) float32
    tet_b2: np.ndarray        # (NT,) float32
    tet_fiber: np.ndarray | None  # (NT,4) float32 f0.xyz, tendonmask
    vert_ntiles: np.ndarray   # (NV,) int32 tiles touching each vertex (new order)
    orphans: np.ndarray       # vertices in no tet (new order)
    materials: list           # list of dicts (XpbdMaterial fields)
    tet_material: np.ndarray  # (NT,) material id per new tet
    tile_own: np.ndarray | None = None  # (n_tiles+1,) tile k owns new ids [tile_own[k], tile_own[k+1])
    tile_group: np.ndarray | None = None  # (n_tiles,) group of each tile when built with vert_group

    @property
    def n_tiles(self) -> int:
        return int(self.tile_nint.shape[0])

    @property
    def n_boundary(self) -> int:
        return int(self.bnd_verts.shape[0])


def ctas_per_sm(materials: list[dict]) -> int:
    """Resident CTAs per SM of the tile pass the library launches for these
    materials: 3 for the light constraint set (ARAP-SVD / aniso only, no
    damping), 2 when any material has volume, SNH or damping."""
    u = 0
    for m in materials:
        u |= int(m["flags"])
    return 2 if u & (capi.MAT_VOLUME | capi.MAT_SNH | capi.MAT_DAMPED) else 3


def default_tile_tets(n_tets: int, n_sm: int = 148, ctas: int = 3, max_tile: int = 2048) -> int:
    """Tile size that fills whole waves: the tile count is a multiple of the
    resident CTA slots (n_sm x ctas) with tiles of at most ``max_tile`` tets,
    so no wave runs part-empty (at least 64 tets per tile)."""
    slots = n_sm * ctas
    waves = max(1, int(np.ceil(n_tets / float(slots * max_tile))))
    t = int(np.ceil(n_tets / float(slots * waves)))
    return int(np.clip(t, 64, max_tile))


def tet_materials(n_tets: int, tets: np.ndarray, table: ConstraintTable):
    """Per-tet constraint flags/parameters from the reference table, deduplicated
    into a material table.  Returns (materials, material_of_tet, V0_of_tet)."""
    flags = np.zeros(n_tets, np.uint32)
    prm = np.zeros((n_tets, 7), np.float32)  # arap_k, vol_k, vol_damp, aniso_k, snh_mu, snh_lam, snh_damp
    V0 = np.full(n_tets, np.nan, np.float32)
    spec = {
        ConstraintType.TETARAPSVD: (capi.MAT_ARAPSVD, [(0, "k")]),
        ConstraintType.TETVOLUME: (capi.MAT_VOLUME, [(1, "k"), (2, "d")]),
        ConstraintType.TETARAPANISO: (capi.MAT_ANISO, [(3, "k")]),
        ConstraintType.TETSNH: (capi.MAT_SNH, [(4, "k"), (5, "lam"), (6, "d")]),
    }
    for ctype, (off, cnt) in table.cons_ranges.items():
        if ctype == ConstraintType.ATTACH:
            continue
        if ctype not in spec:
            raise NotImplementedError(f"constraint type {ctype.name} is not on the sm_100a path")
        sl = slice(off, off + cnt)
        tid = table.c_tetid[sl]
        if np.unique(tid).shape[0] != tid.shape[0]:
            raise NotImplementedError(f"two {ctype.name} constraints on one tet are not supported")
        if not np.array_equal(table.c_pts[sl], tets[tid]):
            raise ValueError(f"{ctype.name} constraint pts differ from the tet's vertices")
        k = table.c_stiffness[sl]
        live = k > 0  # the reference kernels return at once when stiffness <= 0
        bit, cols = spec[ctype]
        t = tid[live]
        flags[t] |= np.uint32(bit)
        for col, what in cols:
            src = {"k": k, "d": table.c_dampingratio[sl], "lam": table.c_restdir[sl, 0]}[what]
            prm[t, col] = src[live]
        if ctype in (ConstraintType.TETVOLUME, ConstraintType.TETSNH):
            V0[t] = table.c_restlength[sl][live]
    damped = ((flags & capi.MAT_VOLUME) != 0) & (prm[:, 2] > 0) | ((flags & capi.MAT_SNH) != 0) & (prm[:, 6] > 0)
    flags[damped] |= np.uint32(capi.MAT_DAMPED)
    key = np.concatenate([flags.view(np.float32)[:, None], prm], axis=1)
    uniq, mat_of = np.unique(key.view(np.dtype((np.void, key.dtype.itemsize * key.shape[1]))).ravel(),
                             return_inverse=True)
    if uniq.shape[0] > capi.MAX_MATERIALS:
        raise ValueError(f"{uniq.shape[0]} distinct tet materials exceed the limit of {capi.MAX_MATERIALS}")
    mats = []
    for u in uniq:
        row = np.frombuffer(u.tobytes(), np.float32)
        mats.append(dict(flags=int(row[:1].view(np.uint32)[0]), arap_k=float(row[1]), vol_k=float(row[2]),
                         vol_damp=float(row[3]), aniso_k=float(row[4]), snh_mu=float(row[5]), snh_lam=float(row[6]),
                         snh_damp=float(row[7])))
    return mats, mat_of.astype(np.int32).ravel(), V0


# Relative projection cost of a tet by constraint (the polar iteration of
# ARAP-SVD dominates; the shared loads, deformation gradient and
# accumulation are the base), from instruction counts of the tile pass.
_COST_BASE, _COST = 0.35, {capi.MAT_ARAPSVD: 0.65, capi.MAT_SNH: 0.35, capi.MAT_VOLUME: 0.15, capi.MAT_ANISO: 0.25}


def tet_cost(materials: list[dict], mat_of_tet: np.ndarray) -> np.ndarray:
    """Estimated relative cost of projecting each tet (1.0 for an ARAP-SVD tet)."""
    mc = np.array([_COST_BASE + sum(c for bit, c in _COST.items() if int(m["flags"]) & bit) for m in materials])
    return mc[mat_of_tet]


def fiber_f0(v_fiber: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """Normalised mean fiber direction per tet in float32, in the order of
    solve_tet_aniso_arap_kernel (solve_kernels.py:1348-1353); zero where the
    mean vanishes (the kernel then skips the tet)."""
    vf = v_fiber.astype(np.float32)
    f = (((vf[tets[:, 0]] + vf[tets[:, 1]]) + vf[tets[:, 2]]) + vf[tets[:, 3]]) / np.float32(4.0)
    fn = np.sqrt(f[:, 0] * f[:, 0] + f[:, 1] * f[:, 1] + f[:, 2] * f[:, 2])
    ok = fn >= np.float32(1e-9)
    out = np.zeros_like(f)
    out[ok] = f[ok] / fn[ok, None]
    return out


def _grouped_codes(x: np.ndarray, group: np.ndarray | None, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """Morton codes over the whole box, or with ``group``: (group, Morton
    code over the group's own box), so each group stays contiguous."""
    if group is None:
        return morton_codes(x, lo, hi)
    ng = int(group.max()) + 1
    glo = np.full((ng, 3), np.inf, np.float64)
    ghi = np.full((ng, 3), -np.inf, np.float64)
    np.minimum.at(glo, group, x)
    np.maximum.at(ghi, group, x)
    codes = morton_codes(x.astype(np.float64), glo[group], ghi[group])
    return (group.astype(np.uint64) << np.uint64(30)) | codes


def build_layout(pos0: np.ndarray, tets: np.ndarray, table: ConstraintTable, *, tile_tets: int | None = None,
                 v_fiber: np.ndarray | None = None, tet_tendonmask: np.ndarray | None = None,
                 n_sm: int = 148, vert_group: np.ndarray | None = None) -> TileLayout:
    """``vert_group`` (optional, per vertex): independent meshes packed in one
    vertex set (batched instances).  Tets are then ordered by group first and
    no tile spans two groups, so any run of whole groups is a closed set of
    tiles (no shared vertices with the other tiles)."""
    pos0 = np.asarray(pos0, np.float32)
    tets = np.asarray(tets, np.int64)
    nv, nt = pos0.shape[0], tets.shape[0]
    if nt == 0:
        raise ValueError("mesh has no tets")
    mats, mat_of_user_tet, V0 = tet_materials(nt, tets, table)
    if tile_tets is None:
        tile_tets = default_tile_tets(nt, n_sm, ctas_per_sm(mats))
    lo, hi = pos0.min(0), pos0.max(0)
    vgroup = None if vert_group is None else np.asarray(vert_group, np.int64)
    tgroup = None if vgroup is None else vgroup[tets[:, 0]]
    if tgroup is not None and not (vgroup[tets] == tgroup[:, None]).all():
        raise ValueError("a tet spans two vertex groups")
    # 1. tets in Morton order of their centroid (within their group)
    cent = pos0[tets].mean(axis=1)
    tet_perm = np.argsort(_grouped_codes(cent, tgroup, lo, hi), kind="stable")
    tet_inv = np.empty(nt, np.int64)
    tet_inv[tet_perm] = np.arange(nt)
    tets_s = tets[tet_perm]
    # 2. tiles of consecutive tets (cut at group starts), as many as equal
    # counts of tile_tets give, cut at equal shares of the estimated projection
    # cost so that tiles holding dearer constraint sets (the aniso muscle's
    # fiber term, volume) hold fewer tets and all tiles reach the per-iteration
    # grid barrier together; split any tile whose vertex set would not fit
    cost = tet_cost(mats, mat_of_user_tet[tet_perm])
    ccum = np.r_[0.0, np.cumsum(cost)]

    def cut(a: int, b: int, k: int) -> list[int]:
        share = ccum[a] + (ccum[b] - ccum[a]) * np.arange(1, k) / k
        inner = np.clip(np.searchsorted(ccum, share, side="left"), a + 1, b - 1) if k > 1 else []
        return [int(x) for x in inner] + [b]

    if tgroup is None:
        bounds = [0] + cut(0, nt, int(np.ceil(nt / tile_tets)))
    else:
        gs = tgroup[tet_perm]
        starts = np.r_[0, np.nonzero(np.diff(gs))[0] + 1, nt]
        bounds = [0]
        for a, b in zip(starts[:-1], starts[1:]):
            bounds += cut(int(a), int(b), int(np.ceil((b - a) / tile_tets)))
    bounds = sorted(set(bounds))
    tptr = [0]
    for a, b in zip(bounds[:-1], bounds[1:]):
        s = a
        while s < b:
            e = b
            while np.unique(tets_s[s:e]).shape[0] > capi.MAX_TILE_VERTS:
                e = s + (e - s) // 2
            tptr.append(e)
            s = e
    tile_tptr = np.asarray(tptr, np.int64)
    n_tiles = tile_tptr.shape[0] - 1
    # Interleave each tile: storage slot j holds the tile's Morton-order tet
    # (j % 32) * ceil(n/32) + j // 32, so the 32 lanes of a warp project tets
    # spread over the whole tile instead of 32 neighbours sharing vertices
    # (which would serialise their shared-memory atomics).
    inter = np.empty(nt, np.int64)
    for a, b in zip(tile_tptr[:-1], tile_tptr[1:]):
        n = int(b - a)
        cols = (n + 31) // 32
        k = np.arange(32 * cols).reshape(cols, 32).T.reshape(-1)  # column-major walk
        k = k[k < n]
        inter[a:b] = a + k
    tet_perm = tet_perm[inter]
    tet_inv[tet_perm] = np.arange(nt)
    tets_s = tets[tet_perm]
    tile_of_tet = np.repeat(np.arange(n_tiles), np.diff(tile_tptr))
    # 3. unique (tile, vertex) pairs
    slot_tile = np.repeat(tile_of_tet, 4)
    slot_v = tets_s.reshape(-1)
    keys = slot_tile * nv + slot_v
    ukeys, slot_u = np.unique(keys, return_inverse=True)
    u_tile, u_v = ukeys // nv, ukeys % nv
    ntile_of_v = np.bincount(u_v, minlength=nv)
    first_tile = np.full(nv, n_tiles, np.int64)
    np.minimum.at(first_tile, u_v, u_tile)
    bnd = ntile_of_v > 1
    # 4. vertex renumbering: (first tile, interior before boundary, Morton)
    vm = _grouped_codes(pos0, vgroup, lo, hi)
    perm = np.lexsort((vm, bnd.astype(np.int64), first_tile))
    inv = np.empty(nv, np.int64)
    inv[perm] = np.arange(nv)
    # 5. per-tile vertex lists (interior first), local slot indices
    u_new = inv[u_v]
    u_bnd = bnd[u_v].astype(np.int64)
    order = np.lexsort((u_new, u_bnd, u_tile))
    pos_of_u = np.empty_like(order)
    pos_of_u[order] = np.arange(order.shape[0])
    tile_verts = u_new[order].astype(np.int32)
    counts = np.bincount(u_tile, minlength=n_tiles)
    tile_vptr = np.zeros(n_tiles + 1, np.int64)
    tile_vptr[1:] = np.cumsum(counts)
    tile_nint = np.bincount(u_tile[u_bnd == 0], minlength=n_tiles)
    local = (pos_of_u[slot_u] - tile_vptr[slot_tile]).reshape(nt, 4)
    max_tile_verts = int(counts.max())
    assert max_tile_verts <= capi.MAX_TILE_VERTS and local.max() < 65536
    # 6. materials, rest data, tet streams
    B, V0_geo, _ = tet_rest_data(pos0, tets)
    V0 = np.where(np.isnan(V0), V0_geo, V0).astype(np.float32)
    Bs = B[tet_perm].reshape(nt, 9)
    tet_q = np.zeros((nt, 4), np.uint32)
    tet_q[:, 0] = (local[:, 0] | (local[:, 1] << 16)).astype(np.uint32)
    tet_q[:, 1] = (local[:, 2] | (local[:, 3] << 16)).astype(np.uint32)
    tet_q[:, 2] = mat_of_user_tet[tet_perm].astype(np.uint32)
    tet_q[:, 3] = V0[tet_perm].view(np.uint32)
    tet_b0 = np.ascontiguousarray(Bs[:, 0:4])
    tet_b1 = np.ascontiguousarray(Bs[:, 4:8])
    tet_b2 = np.ascontiguousarray(Bs[:, 8])
    tet_fiber = None
    if any(m["flags"] & capi.MAT_ANISO for m in mats):
        if v_fiber is None:
            raise ValueError("aniso_arap needs per-vertex fiber directions")
        f0 = fiber_f0(v_fiber, tets)
        tm = np.zeros(nt, np.float32) if tet_tendonmask is None else np.asarray(tet_tendonmask, np.float32)
        tet_fiber = np.concatenate([f0, tm[:, None]], axis=1)[tet_perm].astype(np.float32)
    return TileLayout(
        n_verts=nv, n_tets=nt, perm=perm, inv=inv, tet_perm=tet_perm, tet_inv=tet_inv,
        tets_new=inv[tets_s].astype(np.int32),
        tile_vptr=tile_vptr.astype(np.int32), tile_nint=tile_nint.astype(np.int32),
        tile_tptr=tile_tptr.astype(np.int32), tile_verts=tile_verts,
        bnd_verts=np.nonzero((ntile_of_v != 1)[perm])[0].astype(np.int32), max_tile_verts=max_tile_verts,
        tet_q=tet_q, tet_b0=tet_b0, tet_b1=tet_b1, tet_b2=tet_b2, tet_fiber=tet_fiber,
        vert_ntiles=ntile_of_v[perm].astype(np.int32), orphans=np.nonzero(ntile_of_v[perm] == 0)[0].astype(np.int32),
        materials=mats, tet_material=mat_of_user_tet[tet_perm].astype(np.int32),
        tile_own=np.searchsorted(first_tile[perm], np.arange(n_tiles + 1)).astype(np.int32),
        tile_group=None if tgroup is None else tgroup[tet_perm][tile_tptr[:-1]].astype(np.int32))
