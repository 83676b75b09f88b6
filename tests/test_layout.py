"""Host-side setup: constraint table, Morton tiles, materials (no GPU)."""
import numpy as np
import pytest

from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.builder import collect_raw_constraints, lumped_mass, tet_rest_data
from rlmusclev2_b200.defs import ConstraintType
from rlmusclev2_b200.layout import build_layout, fiber_f0
from tests._cases import CFG1_CONSTRAINTS, cfg1_mesh
from oracle import oracle as O


def _reconstruct(L):
    loc = np.stack([L.tet_q[:, 0] & 0xFFFF, L.tet_q[:, 0] >> 16, L.tet_q[:, 1] & 0xFFFF, L.tet_q[:, 1] >> 16],
                   1).astype(np.int64)
    tile_of = np.repeat(np.arange(L.n_tiles), np.diff(L.tile_tptr))
    return L.tile_verts[L.tile_vptr[tile_of][:, None] + loc]


@pytest.mark.parametrize("tile_tets", [64, 256, 2048])
def test_tiles_reconstruct_mesh(tile_tets):
    m = cfg1_mesh()
    t = collect_raw_constraints(m.verts, m.tets, CFG1_CONSTRAINTS).sorted_by_type()
    L = build_layout(m.verts, m.tets, t, tile_tets=tile_tets)
    assert np.array_equal(_reconstruct(L), L.tets_new)
    assert np.array_equal(L.perm[L.tets_new], m.tets[L.tet_perm])
    # interior vertices are touched by exactly one tile, boundary by several
    owners = np.zeros(m.verts.shape[0], np.int64)
    for ti in range(L.n_tiles):
        vs = np.unique(L.tets_new[L.tile_tptr[ti]:L.tile_tptr[ti + 1]])
        owners[vs] += 1
        lst = L.tile_verts[L.tile_vptr[ti]:L.tile_vptr[ti + 1]]
        assert set(lst.tolist()) == set(vs.tolist())
        assert np.all(owners[lst[:L.tile_nint[ti]]] >= 1)
    bnd = set(L.bnd_verts.tolist())
    for ti in range(L.n_tiles):
        lst = L.tile_verts[L.tile_vptr[ti]:L.tile_vptr[ti + 1]]
        nint = L.tile_nint[ti]
        assert all(owners[v] == 1 and v not in bnd for v in lst[:nint])
        assert all(owners[v] > 1 and v in bnd for v in lst[nint:])
    assert L.max_tile_verts <= capi.MAX_TILE_VERTS


def test_table_sorted_like_reference():
    m = cfg1_mesh()
    t = collect_raw_constraints(m.verts, m.tets, CFG1_CONSTRAINTS).sorted_by_type()
    assert list(t.cons_ranges) == [ConstraintType.TETVOLUME, ConstraintType.TETARAPSVD]
    assert t.cons_ranges[ConstraintType.TETVOLUME] == (0, 12288)
    assert np.all(np.diff(t.c_type) >= 0)
    assert np.isinf(t.c_stiffness[0]) and t.c_stiffness[-1] == np.float32(1e7)


def test_rest_data_matches_oracle():
    m = cfg1_mesh()
    B, V0, valid = tet_rest_data(m.verts, m.tets)
    rv, Bo, mass_o, tot = O.precompute_rest(m.verts, m.tets, 1060.0, "f64")
    np.testing.assert_allclose(B, Bo, rtol=1e-5, atol=1e-2)
    np.testing.assert_allclose(np.abs(V0), rv, rtol=1e-6)
    mass, vol = lumped_mass(m.verts, m.tets, 1060.0)
    np.testing.assert_allclose(mass, mass_o, rtol=1e-6)
    assert valid.all() and (V0 > 0).all()


def test_materials_dedup_and_flags():
    m = cfg1_mesh()
    cfg = CFG1_CONSTRAINTS + [{"type": "snh", "name": "snh", "mu": 2e4, "lam": 1e6, "dampingratio": 0.1}]
    mask = np.zeros(m.tets.shape[0], bool)
    mask[:100] = True
    t = collect_raw_constraints(m.verts, m.tets, cfg, tet_masks={"snh": mask}).sorted_by_type()
    L = build_layout(m.verts, m.tets, t)
    flags = sorted(mm["flags"] for mm in L.materials)
    base = capi.MAT_ARAPSVD | capi.MAT_VOLUME
    assert flags == [base, base | capi.MAT_SNH | capi.MAT_DAMPED]


def test_fiber_f0_normalised():
    m = cfg1_mesh()
    vf = np.tile(np.array([[0, 0, 1]], np.float32), (m.verts.shape[0], 1))
    f0 = fiber_f0(vf, m.tets)
    np.testing.assert_allclose(f0, np.tile([0, 0, 1], (m.tets.shape[0], 1)), atol=1e-7)
