"""Argument checks of the C ABI run before any launch, so they are testable
without a GPU: every entry point rejects null pointers, bad sizes and
misaligned buffers with a negative code and a message."""
import ctypes as C

import pytest

from rlmusclev2_b200 import _capi as capi

ERR_ARG, ERR_ALIGN, ERR_LIMIT = -1, -2, -4


@pytest.fixture(scope="module")
def lib():
    return capi.load()


def _msg(lib):
    m = lib.xpbd_error_string()
    return m.decode() if m else ""


def test_gemm_rejects_bad_shapes(lib):
    g = capi.XpbdGemm()
    assert lib.xpbd_gemm_bf16(C.byref(g), 256, None) == ERR_ARG          # null operands
    g.a, g.b = 16, 16                                                  # aligned dummies, never dereferenced
    g.m, g.n, g.k, g.lda, g.ldb = 128, 256, 100, 128, 128
    assert lib.xpbd_gemm_bf16(C.byref(g), 256, None) == ERR_ARG          # k % 64 != 0
    assert "k % 64" in _msg(lib)
    g.k = 128
    assert lib.xpbd_gemm_bf16(C.byref(g), 24, None) == ERR_ARG           # n_tile not a multiple of 16
    g.lda = 130
    assert lib.xpbd_gemm_bf16(C.byref(g), 256, None) == ERR_ARG          # lda not a multiple of 8
    g.lda, g.a = 128, 8
    assert lib.xpbd_gemm_bf16(C.byref(g), 256, None) == ERR_ALIGN        # misaligned operand


def test_persistent_and_batched_checks(lib):
    prm, tiles, verts, ps = capi.XpbdParams(), capi.XpbdTiles(), capi.XpbdVerts(), capi.XpbdPersist()
    assert lib.xpbd_iterate_persistent(None, None, None, None, 1, None) == ERR_ARG
    assert lib.xpbd_iterate_persistent(C.byref(prm), C.byref(tiles), C.byref(verts), C.byref(ps), -1, None) == ERR_ARG
    assert lib.xpbd_iterate_persistent(C.byref(prm), C.byref(tiles), C.byref(verts), C.byref(ps), 0, None) == 0
    assert lib.xpbd_iterate_persistent(C.byref(prm), C.byref(tiles), C.byref(verts), C.byref(ps), 2, None) == ERR_ARG
    sb = capi.XpbdSdfBatch()
    assert lib.xpbd_sdf_bake_capsules_batched(C.byref(sb), 2, None, None, C.c_float(0.01), None) == ERR_ARG
    assert lib.xpbd_vertex_step_batched(C.byref(prm), C.byref(verts), capi.OP_SDF, None, None) < 0


def test_learned_glue_checks(lib):
    cf = capi.XpbdCageFeatures()
    assert lib.xpbd_cage_features(C.byref(cf), None, None, None, None, None) == ERR_ARG
    assert lib.xpbd_cage_apply(0, None, None, None, 16, C.c_float(1.0), None, None) == ERR_ARG
    assert lib.xpbd_fallback_select(10, None, None, C.c_float(2.0), None, None, None, None) == ERR_ARG
    assert lib.xpbd_adam(0, 0, None, None, 0, None, None, C.c_float(1e-3), C.c_float(0.9), C.c_float(0.999),
                         C.c_float(1e-8), 1, None, None, 0, None) == ERR_ARG
    assert lib.xpbd_mse_grad(0, 0, 3, 64, None, 16, None, 3, None, None, 0, None, None) == ERR_ARG


def test_noalloc_rejects_oversized_meshes(lib):
    prm, tiles, verts = capi.XpbdParams(), capi.XpbdTiles(), capi.XpbdVerts()
    verts.n = capi.NOALLOC_MAX_VERTS + 1
    assert lib.xpbd_iterate_noalloc(C.byref(prm), C.byref(tiles), C.byref(verts), None) == ERR_LIMIT
    assert "XPBD_NOALLOC_MAX_VERTS" in _msg(lib)


def test_bone_glue_fascia_checks(lib):
    A, M8, M4 = 16, 8, 4  # aligned dummy, 8-byte (not 16), 4-byte (not 8): never dereferenced
    f = C.c_float
    # bone binding
    assert lib.xpbd_bone_bind(-1, A, 3, A, 1, A, f(1.0), A, A, A, None) == ERR_ARG
    assert lib.xpbd_bone_bind(1, A, 3, A, 0, A, f(1.0), A, A, A, None) == ERR_ARG         # no triangles
    assert lib.xpbd_bone_bind(1, M8, 3, A, 1, A, f(1.0), A, A, A, None) == ERR_ALIGN      # query4
    assert lib.xpbd_bone_bind(1, A, 3, A, 1, A, f(1.0), A, M4, A, None) == ERR_ALIGN      # uv
    assert lib.xpbd_bone_bind(0, None, 3, A, 1, A, f(1.0), None, None, None, None) == 0
    # sliding targets: re-projection needs the muscle positions and anchors; some target is required
    assert lib.xpbd_bone_slide_targets(1, None, A, A, A, A, A, f(0.01), 1, f(1.0), 3, A, 1, A, A, A, None) == ERR_ARG
    assert lib.xpbd_bone_slide_targets(1, A, A, A, A, A, A, f(0.01), 0, f(1.0), 3, A, 1, A, None, None,
                                       None) == ERR_ARG
    assert lib.xpbd_bone_slide_targets(1, A, A, A, A, A, A, f(0.01), 0, f(1.0), 3, A, 1, A, M8, None,
                                       None) == ERR_ALIGN
    assert lib.xpbd_bone_slide_targets(0, None, None, None, None, None, None, f(0.01), 0, f(1.0), 3, A, 1, A,
                                       None, None, None) == 0
    assert lib.xpbd_bone_surface_pose(4, A, A, 0, A, A, None) == ERR_ARG                  # no bones
    assert lib.xpbd_bone_surface_pose(4, A, A, 2, A, M8, None) == ERR_ALIGN
    # fascia ride
    assert lib.xpbd_surface_bind(1, A, 3, A, 0, A, f(1.0), A, A, A, A, None) == ERR_ARG
    assert lib.xpbd_surface_bind(1, A, 3, A, 1, A, f(1.0), A, M4, A, A, None) == ERR_ALIGN
    assert lib.xpbd_surface_ride(1, A, A, A, A, M8, A, A, None) == ERR_ALIGN
    assert lib.xpbd_surface_ride(0, None, None, None, None, None, None, None, None) == 0
    # fascia squeeze
    assert lib.xpbd_fascia_advect(1, None, A, A, A, None) == ERR_ARG
    assert lib.xpbd_fascia_advect(1, A, A, M8, A, None) == ERR_ALIGN
    assert lib.xpbd_fascia_advect(0, None, None, None, None, None) == 0
    assert lib.xpbd_fascia_anchor(1, A, None, A, A, A, None) == ERR_ARG
    assert lib.xpbd_fascia_anchor(1, A, A, A, A, M8, None) == ERR_ALIGN
    assert lib.xpbd_fascia_glue(1, A, A, A, A, A, A, f(0.0), f(1.0), None) == ERR_ARG      # dt <= 0
    assert lib.xpbd_fascia_glue(1, A, A, A, A, A, M8, f(0.01), f(1.0), None) == ERR_ALIGN
    # muscle-to-muscle glue
    assert lib.xpbd_m2m_glue(1, A, A, A, A, A, f(-1.0), f(1.0), None) == ERR_ARG
    assert lib.xpbd_m2m_glue(1, A, A, A, A, M8, f(0.01), f(1.0), None) == ERR_ALIGN
    assert lib.xpbd_m2m_glue(0, None, None, None, None, None, f(0.01), f(1.0), None) == 0


def test_dcd_checks(lib):
    sz = capi.XpbdDcdWorkspaceSizes()
    assert lib.xpbd_dcd_workspace_query(0, C.byref(sz)) == ERR_ARG
    assert lib.xpbd_dcd_workspace_query(1000, C.byref(sz)) == 0
    assert sz.hist > 4 and sz.split >= 4 and sz.keys == 1000   # the sort's 4 barrier words end ws_hist
    assert lib.xpbd_dcd_broadphase(None, 16, 0, None) == ERR_ARG
    d = capi.XpbdDcd()
    d.n_tris, d.n_verts, d.max_pairs, d.max_contacts = 10, 12, 64, 64
    for name, typ in capi.XpbdDcd._fields_:
        if typ is C.c_void_p:
            setattr(d, name, 16)                                   # aligned dummies, never dereferenced
    assert lib.xpbd_dcd_broadphase(C.byref(d), 8, 0, None) == ERR_ARG    # pos4 misaligned
    d.max_pairs = 0
    assert lib.xpbd_dcd_broadphase(C.byref(d), 16, 0, None) == ERR_ARG   # no pair capacity
    d.max_pairs, d.ws_split = 64, 8
    assert lib.xpbd_dcd_broadphase(C.byref(d), 16, 0, None) == ERR_ALIGN
    d.ws_split, d.tris = 16, None
    assert lib.xpbd_dcd_narrow_respond(C.byref(d), 16, None) == ERR_ARG


def test_blend_to_target_checks(lib):
    f = lib.xpbd_blend_to_target
    assert f(-1, None, 4, None, None, C.c_float(0.5), None) == ERR_ARG           # negative count
    assert f(8, None, 4, 16, 16, C.c_float(0.5), None) == ERR_ARG                # n > n_verts without idx
    assert f(2, None, 4, None, 16, C.c_float(0.5), None) == ERR_ARG              # null positions
    assert f(2, None, 4, 16, 16, C.c_float(float("nan")), None) == ERR_ARG     # non-finite beta
    assert "beta" in _msg(lib)
    assert f(2, None, 4, 8, 16, C.c_float(0.5), None) == ERR_ALIGN               # misaligned positions
    assert f(0, None, 4, 16, 16, C.c_float(0.5), None) == 0                      # nothing to do
    assert f(2, None, 4, 16, 16, C.c_float(0.0), None) == 0                      # beta 0: no launch


def test_svd_clamp_checks(lib):
    tiles, verts = capi.XpbdTiles(), capi.XpbdVerts()
    assert lib.xpbd_svd_clamp(None, None, C.c_float(0.1), C.c_float(1.0), 1, None) == ERR_ARG
    assert lib.xpbd_svd_clamp(C.byref(tiles), C.byref(verts), C.c_float(0.1), C.c_float(1.0), 1, None) == ERR_ARG


def test_multigrid_transfer_checks(lib):
    g = capi.XpbdCage()
    assert lib.xpbd_mg_coarse_reset(None, None, 16, None, None, None) == ERR_ARG      # no cage
    assert lib.xpbd_mg_coarse_reset(C.byref(g), None, 16, None, None, None) == ERR_ARG  # empty cage
    g.n_fine, g.n_coarse, g.n_blocks, g.max_block = 8, 4, 1, 4
    for k in ("r_ptr", "r_fine", "r_w", "blk_ptr", "blk_moff", "minv", "coarse_lib", "p_idx", "p_w", "resid", "rhs"):
        setattr(g, k, 16)  # aligned dummies, never dereferenced
    assert lib.xpbd_mg_coarse_reset(C.byref(g), None, None, None, None, None) == ERR_ARG
    assert "null coarse" in _msg(lib)
    assert lib.xpbd_mg_coarse_reset(C.byref(g), 32, 32, None, None, None) == ERR_ARG  # src aliases coarse
    assert lib.xpbd_mg_coarse_reset(C.byref(g), 40, 32, None, None, None) == ERR_ALIGN
    assert lib.xpbd_mg_coarse_reset(C.byref(g), None, 32, 8, None, None) == ERR_ALIGN
    assert lib.xpbd_mg_restrict(C.byref(g), None, 32, None, None, None) == ERR_ARG
    assert lib.xpbd_mg_prolong_delta(C.byref(g), 32, None, 24, None, None, None) == ERR_ALIGN
