"""The allocation-free iteration (xpbd_iterate_noalloc) against the regular one.

Callers that cannot allocate device memory -- a step recorded inside someone
else's CUDA graph capture, a plugin whose host owns all GPU memory, a
real-time loop -- use xpbd_iterate_noalloc, whose Jacobi accumulator is a
fixed device array inside the library.  Two engines start from the same
state; one iterates through xpbd_project + xpbd_apply_boundary with its own
accumulator, the other through xpbd_iterate_noalloc; after each of two calls
in a row the positions agree to the parity tolerance (1e-5 x bbox diagonal;
only the order of the float atomics differs).  This file is collected last so
that a failure here does not hide the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from rlmusclev2_b200 import MuscleSim
from rlmusclev2_b200 import _capi as capi
from tests._cases import CFG1, CFG1_CONSTRAINTS, bbox_diag, cfg1_mesh

pytestmark = pytest.mark.gpu


def _sim(m):
    return MuscleSim.from_procedural(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                                     device="cuda:0", stopped=m.stopped, **CFG1)


def test_noalloc_iteration_matches_regular_two_calls():
    m = cfg1_mesh()
    a, b = _sim(m), _sim(m)
    for s in (a, b):
        s.integrate()  # a predicted state with something to project
    lib = capi.load()
    tol = 1e-5 * bbox_diag(m.verts)
    for call in range(2):
        capi.check(lib.xpbd_project(C.byref(a._prm), C.byref(a._tiles), C.byref(a._verts), capi.PROJECT_FUSED, a._sp))
        capi.check(lib.xpbd_apply_boundary(C.byref(a._prm), C.byref(a._tiles), C.byref(a._verts),
                                           capi.APPLY_ATTACH | capi.APPLY_DIVIDE | capi.APPLY_PIN | capi.APPLY_CLEAR,
                                           a._sp))
        capi.check(lib.xpbd_iterate_noalloc(C.byref(b._prm), C.byref(b._tiles), C.byref(b._verts), b._sp))
        pa, pb = a.positions_np(), b.positions_np()
        err = np.abs(pa - pb).max()
        moved = np.abs(pa - m.verts).max()
        print(f"call {call}: max |noalloc - regular| = {err:.3e} (tol {tol:.3e}, moved {moved:.3e})")
        assert moved > 10 * tol
        assert err <= tol


def test_noalloc_rejects_oversized_mesh():
    m = cfg1_mesh()
    s = _sim(m)
    v = capi.XpbdVerts()
    C.memmove(C.addressof(v), C.addressof(s._verts), C.sizeof(v))
    v.n = capi.NOALLOC_MAX_VERTS + 1
    rc = capi.load().xpbd_iterate_noalloc(C.byref(s._prm), C.byref(s._tiles), C.byref(v), s._sp)
    assert rc == -4  # XPBD_ERR_LIMIT
    assert b"XPBD_NOALLOC_MAX_VERTS" in capi.load().xpbd_error_string()
