"""ctypes binding of libxpbd_b200.so (include/xpbd_b200.h).

The library is the product's only compute path: importing this module on a
machine with a GPU and no built library raises instead of falling back to any
Python or CPU implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

MAX_MATERIALS = 64
MAX_ATTACH_MATERIALS = 16
MAX_TILE_VERTS = 4096
NOALLOC_MAX_VERTS = 262144

OK = 0
MAT_ARAPSVD, MAT_VOLUME, MAT_ANISO, MAT_SNH, MAT_DAMPED = 1, 2, 4, 8, 16
VF_ATTACH_MASK, VF_PIN = 0xFF, 1 << 8
OP_SDF, OP_VELOCITY, OP_PREDICT, OP_PIN = 1, 2, 4, 8
STATUS_PAIR_OVERFLOW, STATUS_CONTACT_OVERFLOW, STATUS_STACK_OVERFLOW, STATUS_BARRIER_TIMEOUT = 1, 2, 4, 8
STATUS_MMA_TIMEOUT = 16
STATUS_ACC_RANGE = 32
APPLY_ATTACH, APPLY_DIVIDE, APPLY_PIN, APPLY_CLEAR = 1, 2, 4, 8
PROJECT_FUSED, PROJECT_ACCUMULATE, PROJECT_FUSED_LAST = 0, 1, 2


class XpbdMaterial(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("arap_k", C.c_float), ("vol_k", C.c_float), ("vol_damp", C.c_float),
                ("aniso_k", C.c_float), ("snh_mu", C.c_float), ("snh_lam", C.c_float), ("snh_damp", C.c_float)]


class XpbdAttachMaterial(C.Structure):
    _fields_ = [("k", C.c_float), ("damp", C.c_float)]


class XpbdParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("gravity", C.c_float * 3), ("veldamping", C.c_float),
                ("quasi_static", C.c_int32), ("omega", C.c_float), ("contraction_ratio", C.c_float),
                ("fiber_stiffness_scale", C.c_float), ("n_materials", C.c_int32),
                ("n_attach_materials", C.c_int32), ("tile_variant", C.c_int32), ("acc_scale", C.c_float),
                ("arap_skip_ssq", C.c_float), ("status", C.c_void_p),
                ("materials", XpbdMaterial * MAX_MATERIALS),
                ("attach", XpbdAttachMaterial * MAX_ATTACH_MATERIALS)]


class XpbdVerts(C.Structure):
    _fields_ = [("n", C.c_int32), ("reserved", C.c_int32), ("pos", C.c_void_p), ("pprev", C.c_void_p),
                ("vel", C.c_void_p), ("mass", C.c_void_p), ("force", C.c_void_p), ("accum", C.c_void_p),
                ("vflags", C.c_void_p), ("attach_target", C.c_void_p), ("pin_target", C.c_void_p)]


class XpbdTiles(C.Structure):
    _fields_ = [("n_tets", C.c_int32), ("n_tiles", C.c_int32), ("n_boundary", C.c_int32),
                ("max_tile_verts", C.c_int32), ("tile_vptr", C.c_void_p), ("tile_nint", C.c_void_p),
                ("tile_tptr", C.c_void_p), ("tile_verts", C.c_void_p), ("tet_q", C.c_void_p),
                ("tet_b0", C.c_void_p), ("tet_b1", C.c_void_p), ("tet_b2", C.c_void_p),
                ("tet_fiber", C.c_void_p), ("tet_act", C.c_void_p), ("bnd_verts", C.c_void_p),
                ("vert_ntiles", C.c_void_p), ("arrive", C.c_void_p)]


class XpbdSdf(C.Structure):
    _fields_ = [("phi", C.c_void_p), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("origin", C.c_float * 3), ("h", C.c_float), ("contact_offset", C.c_float),
                ("max_push", C.c_float), ("reserved", C.c_int32)]


class XpbdCapsule(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("half", C.c_float), ("axis", C.c_float * 3), ("radius", C.c_float)]


class XpbdCage(C.Structure):
    _fields_ = [("n_fine", C.c_int32), ("n_coarse", C.c_int32), ("n_blocks", C.c_int32), ("max_block", C.c_int32),
                ("r_ptr", C.c_void_p), ("r_fine", C.c_void_p), ("r_w", C.c_void_p), ("blk_ptr", C.c_void_p),
                ("blk_moff", C.c_void_p), ("minv", C.c_void_p), ("coarse_lib", C.c_void_p), ("p_idx", C.c_void_p),
                ("p_w", C.c_void_p), ("resid", C.c_void_p), ("rhs", C.c_void_p)]


class XpbdDcd(C.Structure):
    _fields_ = [("n_tris", C.c_int32), ("n_verts", C.c_int32), ("max_pairs", C.c_int32), ("max_contacts", C.c_int32),
                ("tris", C.c_void_p), ("tri_group", C.c_void_p), ("allow_self", C.c_int32),
                ("jacobi_avg", C.c_int32), ("thickness", C.c_float), ("offset_eps", C.c_float),
                ("multiplier", C.c_float), ("friction_static", C.c_float), ("friction_dynamic", C.c_float),
                ("max_push", C.c_float), ("box_lo", C.c_float * 3), ("box_hi", C.c_float * 3),
                ("pairs", C.c_void_p), ("n_pairs", C.c_void_p), ("n_contacts", C.c_void_p), ("c_ids", C.c_void_p),
                ("c_data", C.c_void_p), ("x_prev", C.c_void_p), ("dP", C.c_void_p), ("status", C.c_void_p),
                ("ws_nodes", C.c_void_p), ("ws_keys", C.c_void_p), ("ws_vals", C.c_void_p),
                ("ws_keys2", C.c_void_p), ("ws_vals2", C.c_void_p), ("ws_hist", C.c_void_p),
                ("ws_bbox", C.c_void_p),
                ("ws_count", C.c_void_p), ("ws_total", C.c_void_p), ("ws_slots", C.c_void_p),
                ("ws_split", C.c_void_p), ("refit_only", C.c_int32)]


class XpbdDcdWorkspaceSizes(C.Structure):
    _fields_ = [("nodes_floats", C.c_int64), ("keys", C.c_int64), ("hist", C.c_int64),
                ("bbox_floats", C.c_int64), ("count", C.c_int64), ("slots", C.c_int64), ("split", C.c_int64)]


class XpbdMetrics(C.Structure):
    _fields_ = [("vol_sum", C.c_double), ("resid_sq_sum", C.c_double), ("resid_max", C.c_float),
                ("n_inverted", C.c_int32), ("n_nonfinite", C.c_int32), ("reserved", C.c_int32)]


class XpbdSdfBatch(C.Structure):
    _fields_ = [("phi", C.c_void_p), ("frame", C.c_void_p), ("vert_inst", C.c_void_p), ("n_inst", C.c_int32),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("contact_offset", C.c_float),
                ("max_push", C.c_float)]


class XpbdGemm(C.Structure):
    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p), ("lda", C.c_int32), ("ldb", C.c_int32), ("m", C.c_int32),
                ("n", C.c_int32), ("k", C.c_int32), ("act", C.c_int32), ("bias", C.c_void_p),
                ("gelu_grad_of", C.c_void_p), ("ld_g", C.c_int32), ("ld_pre", C.c_int32), ("ld_f32", C.c_int32),
                ("ld_bf16", C.c_int32), ("ld_bf16_t", C.c_int32), ("flags", C.c_int32), ("out_pre", C.c_void_p),
                ("out_f32", C.c_void_p), ("out_bf16", C.c_void_p), ("out_bf16_t", C.c_void_p),
                ("status", C.c_void_p)]


class XpbdCageFeatures(C.Structure):
    _fields_ = [("n_cage", C.c_int32), ("m_pad", C.c_int32), ("coarse_lib", C.c_void_p), ("nbr", C.c_void_p),
                ("owner", C.c_void_p), ("act_muscle", C.c_void_p), ("cage_bone", C.c_void_p), ("cage_w", C.c_void_p),
                ("bone_rel", C.c_void_p), ("stat", C.c_void_p), ("c_rest4", C.c_void_p), ("c_target4", C.c_void_p),
                ("norm", C.c_void_p)]


class XpbdPersist(C.Structure):
    _fields_ = [("tile_own", C.c_void_p), ("ring", C.c_void_p), ("sync", C.c_void_p), ("status", C.c_void_p),
                ("tile_begin", C.c_int32), ("tile_end", C.c_int32), ("nbr_ptr", C.c_void_p),
                ("nbr_idx", C.c_void_p), ("tile_cnt", C.c_void_p)]


P = C.c_void_p
_SIGS = {
    "xpbd_abi_version": ([], C.c_int),
    "xpbd_bone_bind": ([C.c_int32, P, C.c_int32, P, C.c_int32, P, C.c_float, P, P, P, P], C.c_int),
    "xpbd_bone_slide_targets": ([C.c_int32, P, P, P, P, P, P, C.c_float, C.c_int32, C.c_float, C.c_int32, P,
                                 C.c_int32, P, P, P, P], C.c_int),
    "xpbd_bone_surface_pose": ([C.c_int32, P, P, C.c_int32, P, P, P], C.c_int),
    "xpbd_m2m_glue": ([C.c_int32, P, P, P, P, P, C.c_float, C.c_float, P], C.c_int),
    "xpbd_surface_bind": ([C.c_int32, P, C.c_int32, P, C.c_int32, P, C.c_float, P, P, P, P, P], C.c_int),
    "xpbd_surface_ride": ([C.c_int32, P, P, P, P, P, P, P, P], C.c_int),
    "xpbd_fascia_advect": ([C.c_int32, P, P, P, P, P], C.c_int),
    "xpbd_fascia_anchor": ([C.c_int32, P, P, P, P, P, P], C.c_int),
    "xpbd_fascia_glue": ([C.c_int32, P, P, P, P, P, P, C.c_float, C.c_float, P], C.c_int),
    "xpbd_acc_scale_for_extent": ([C.c_float], C.c_float),
    "xpbd_error_string": ([], C.c_char_p),
    "xpbd_vertex_step": ([C.POINTER(XpbdParams), C.POINTER(XpbdVerts), C.c_uint32, C.POINTER(XpbdSdf), P], C.c_int),
    "xpbd_project": ([C.POINTER(XpbdParams), C.POINTER(XpbdTiles), C.POINTER(XpbdVerts), C.c_int32, P], C.c_int),
    "xpbd_apply_boundary": ([C.POINTER(XpbdParams), C.POINTER(XpbdTiles), C.POINTER(XpbdVerts), C.c_uint32, P],
                            C.c_int),
    "xpbd_apply_all": ([C.POINTER(XpbdParams), C.POINTER(XpbdVerts), C.c_uint32, P], C.c_int),
    "xpbd_pin_overwrite_masked": ([C.c_int32, P, P, P, P, P, P], C.c_int),
    "xpbd_metrics": ([C.POINTER(XpbdTiles), C.POINTER(XpbdVerts), P, P], C.c_int),
    "xpbd_bone_targets": ([C.c_int32, C.c_int32, P, P, P, P, P, P, P], C.c_int),
    "xpbd_blend_to_target": ([C.c_int32, P, C.c_int32, P, P, C.c_float, P], C.c_int),
    "xpbd_svd_clamp": ([P, P, C.c_float, C.c_float, C.c_int32, P], C.c_int),
    "xpbd_sdf_bake_capsules": ([C.POINTER(XpbdSdf), C.c_int32, P, P, C.c_float, P], C.c_int),
    "xpbd_sdf_bake_capsules_batched": ([C.POINTER(XpbdSdfBatch), C.c_int32, P, P, C.c_float, P], C.c_int),
    "xpbd_vertex_step_batched": ([C.POINTER(XpbdParams), C.POINTER(XpbdVerts), C.c_uint32, C.POINTER(XpbdSdfBatch),
                                  P], C.c_int),
    "xpbd_gather": ([C.c_int32, C.c_int32, P, P, C.c_int32, P, C.c_int32, P], C.c_int),
    "xpbd_mg_restrict": ([C.POINTER(XpbdCage), P, P, P, P, P], C.c_int),
    "xpbd_mg_coarse_reset": ([C.POINTER(XpbdCage), P, P, P, P, P], C.c_int),
    "xpbd_mg_prolong_delta": ([C.POINTER(XpbdCage), P, P, P, P, P, P], C.c_int),
    "xpbd_dcd_workspace_query": ([C.c_int32, C.POINTER(XpbdDcdWorkspaceSizes)], C.c_int),
    "xpbd_dcd_broadphase": ([C.POINTER(XpbdDcd), P, C.c_int32, P], C.c_int),
    "xpbd_dcd_narrow_respond": ([C.POINTER(XpbdDcd), P, P], C.c_int),
    "xpbd_iterate_noalloc": ([C.POINTER(XpbdParams), C.POINTER(XpbdTiles), C.POINTER(XpbdVerts), P], C.c_int),
    "xpbd_iterate_persistent": ([C.POINTER(XpbdParams), C.POINTER(XpbdTiles), C.POINTER(XpbdVerts),
                                 C.POINTER(XpbdPersist), C.c_int32, P], C.c_int),
    "xpbd_persistent_fits": ([C.POINTER(XpbdParams), C.POINTER(XpbdTiles), C.POINTER(C.c_int32),
                              C.POINTER(C.c_int32)], C.c_int),
    "xpbd_gemm_bf16": ([C.POINTER(XpbdGemm), C.c_int32, P], C.c_int),
    "xpbd_colsum_bf16": ([C.c_int32, C.c_int32, P, C.c_int32, P, P], C.c_int),
    "xpbd_adam": ([C.c_int32, C.c_int32, P, P, C.c_int32, P, P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32,
                   P, P, C.c_int32, P], C.c_int),
    "xpbd_mse_grad": ([C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, C.c_int32, P, C.c_int32, P, P, C.c_int32, P, P],
                      C.c_int),
    "xpbd_cage_features": ([C.POINTER(XpbdCageFeatures), P, P, P, P, P], C.c_int),
    "xpbd_cage_apply": ([C.c_int32, P, P, P, C.c_int32, C.c_float, P, P], C.c_int),
    "xpbd_cage_target": ([C.c_int32, P, P, P, C.c_float, P, P], C.c_int),
    "xpbd_fallback_select": ([C.c_int32, P, P, C.c_float, P, P, P, P], C.c_int),
    "xpbd_graph_begin": ([P], C.c_int),
    "xpbd_graph_end": ([P, C.POINTER(C.c_void_p)], C.c_int),
    "xpbd_graph_launch": ([P, P], C.c_int),
    "xpbd_graph_destroy": ([P], C.c_int),
}

_LIB = None


def lib_path() -> Path:
    return Path(__file__).resolve().parent / "lib" / "libxpbd_b200.so"


def load(build_if_missing: bool = False) -> C.CDLL:
    """Load the CUDA library; raise if it is missing (there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not path.exists():
        if build_if_missing:
            from .build import build
            build()
        if not path.exists():
            raise RuntimeError(f"{path} is not built; run `python -m rlmusclev2_b200.build` "
                               "(the XPBD substep has no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


class XpbdError(RuntimeError):
    pass


def check(rc: int) -> None:
    if rc != OK:
        msg = load().xpbd_error_string()
        raise XpbdError(f"libxpbd_b200 error {rc}: {msg.decode() if msg else ''}")
