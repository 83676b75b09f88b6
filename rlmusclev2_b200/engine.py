"""XpbdEngine: the reference's shared substep engine (src/muscle/engine.py:780-1211)
rebuilt on the sm_100a library.

Device state lives in torch tensors in the library's vertex/tet order (Morton
tiles, see layout.py); the public accessors convert to and from the
reference's (user) order at the API boundary.  Every compute step is a call
into libxpbd_b200.so on the engine's own CUDA stream; there is no CPU path.

Primitive methods keep the reference's unfused semantics (``clear`` zeroes
dP/dPw, ``solve_constraints`` accumulates, ``apply_dP`` divides,
``apply_pintotarget`` snaps).  ``run_program``/``step`` use the fused kernels
(one tile pass per Jacobi iteration that also applies interior vertices, one
per-vertex kernel per substep boundary) and replay whole frames as CUDA graphs
when no Python hooks are registered.
"""
from __future__ import annotations

import ctypes as C
import logging

import numpy as np
import torch

from . import _capi as capi
from .builder import ConstraintTable
from .defs import ConstraintType
from .layout import TileLayout, build_layout

log = logging.getLogger(__name__)


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


#: the fixed-point accumulator's per-tet range: a tet whose 12 correction
#: magnitudes sum above half to one times the larger of ACC_RANGE_EDGES longest
#: rest edges and the largest rest coordinate raises ACC_RANGE
ACC_RANGE_EDGES = 128.0


def max_rest_edge(pos: np.ndarray, tets: np.ndarray) -> float:
    """Longest of the six edges over all tets of a rest mesh."""
    x = np.asarray(pos, np.float64)
    t = np.asarray(tets, np.int64)
    m = 0.0
    for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
        m = max(m, float(np.sqrt(((x[t[:, a]] - x[t[:, b]]) ** 2).sum(1)).max(initial=0.0)))
    return m


def status_error(tile_status: int, dcd_status: int = 0) -> str | None:
    """The error a frame must raise for its status words, or None.

    ``tile_status``: the XPBD_STATUS_* word of the tile passes and the
    persistent pass; ``dcd_status``: the DCD's word.  Fatal: a grid barrier
    that gave up (its later barriers race), a fixed-point correction beyond
    the accumulator's safe range (the sums wrap), a DCD sort that gave up
    (the broadphase finds no pairs until the words are cleared).  Overflow
    bits of the DCD are warnings (UdcfDcdCollider.stats reports them)."""
    msgs = []
    if tile_status & capi.STATUS_BARRIER_TIMEOUT:
        msgs.append("the persistent Jacobi pass gave up waiting at a grid barrier (positions are invalid)")
    if tile_status & capi.STATUS_ACC_RANGE:
        msgs.append("a tet correction left the fixed-point accumulator's range (positions are invalid: "
                    "the state probably diverged or acc_scale is too large)")
    if dcd_status & capi.STATUS_BARRIER_TIMEOUT:
        msgs.append("the DCD broadphase sort gave up waiting at a grid barrier (contacts were skipped)")
    if not msgs:
        return None
    return "; ".join(msgs) + ". The status words have been cleared for the next launch."



class XpbdEngine:
    """State-independent substep primitives plus the program runner."""

    #: fused Jacobi iteration: PROJECT_FUSED (tile pass + boundary finish
    #: launch; measured faster on B200) or PROJECT_FUSED_LAST (one launch)
    fused_mode = capi.PROJECT_FUSED
    #: replay frames as CUDA graphs (False: launch the same kernels eagerly)
    use_graphs = True

    # subclasses fill these before calling _setup_device()
    pos0_np: np.ndarray
    tet_np: np.ndarray
    n_verts: int

    # ------------------------------------------------------------------ setup
    def _setup_device(self, device, *, mass: np.ndarray, stopped: np.ndarray, table: ConstraintTable,
                      v_fiber: np.ndarray | None, tet_tendonmask: np.ndarray | None, dt: float,
                      gravity_vec, veldamping: float, quasi_static: bool, omega: float = 1.0,
                      contraction_ratio: float = 0.0, fiber_stiffness_scale: float = 1.0,
                      tile_tets: int | None = None, stream=None, vert_group: np.ndarray | None = None) -> None:
        self._lib = capi.load()
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("the sm_100a XPBD engine runs on CUDA devices only (no CPU path); "
                               "pass device='cuda:0'")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available")
        self._stream = stream if stream is not None else torch.cuda.Stream(self.device)
        self._sp = C.c_void_p(self._stream.cuda_stream)
        self.table = table
        self.n_cons = table.n
        self.cons_ranges = dict(table.cons_ranges)
        L = build_layout(self.pos0_np, self.tet_np, table, tile_tets=tile_tets, v_fiber=v_fiber,
                         tet_tendonmask=tet_tendonmask,
                         n_sm=torch.cuda.get_device_properties(self.device).multi_processor_count,
                         vert_group=vert_group)
        self.layout: TileLayout = L
        dev = self.device
        f32 = torch.float32

        def T(a, dtype=None):
            return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dtype)

        nv = self.n_verts
        self._mass_user = np.asarray(mass, np.float32)
        self._stopped_user = np.asarray(stopped, np.int32).copy()
        inv_m = self._inv_mass_user()
        p4 = np.zeros((nv, 4), np.float32)
        p4[:, :3] = self.pos0_np
        p4[:, 3] = inv_m
        self._pos4 = T(p4[L.perm])
        self._prev4 = self._pos4.clone()
        v4 = np.zeros((nv, 4), np.float32)
        v4[:, 3] = (self._stopped_user != 0)
        self._vel4 = T(v4[L.perm])
        self._massd = T(self._mass_user[L.perm])
        self._accum = torch.zeros((nv, 4), dtype=f32, device=dev)
        self._accum_dirty = False
        # persistent multi-iteration pass: boundary ring, grid barrier words, status
        self._ring = torch.zeros((3, nv, 4), dtype=f32, device=dev)
        self._psync = torch.zeros(4, dtype=torch.int32, device=dev)
        self._pstatus = torch.zeros(1, dtype=torch.int32, device=dev)
        # host copies of the status words, queued behind every frame (see _post_status)
        self._status_host = torch.zeros(2, dtype=torch.int32).pin_memory()
        self._status_event = None
        self._t_own = T(L.tile_own)
        self.use_persistent = True
        self._metrics_buf = torch.zeros(8, dtype=torch.float64, device=dev)  # >= sizeof(XpbdMetrics)
        # tiles
        self._t_vptr = T(L.tile_vptr)
        self._t_nint = T(L.tile_nint)
        self._t_tptr = T(L.tile_tptr)
        self._t_verts = T(L.tile_verts)
        self._t_q = T(L.tet_q.view(np.int32))
        self._t_b0 = T(L.tet_b0)
        self._t_b1 = T(L.tet_b1)
        self._t_b2 = T(L.tet_b2)
        self._t_fiber = T(L.tet_fiber) if L.tet_fiber is not None else None
        self._t_act = torch.zeros(L.n_tets, dtype=f32, device=dev) if L.tet_fiber is not None else None
        self._t_bnd = T(L.bnd_verts) if L.n_boundary else torch.zeros(1, dtype=torch.int32, device=dev)
        self._t_ntiles = T(L.vert_ntiles)
        self._t_arrive = torch.zeros(nv, dtype=torch.int32, device=dev)
        self._t_orph = T(L.orphans) if L.orphans.shape[0] else None
        # vertex constraints (attach, pin) in library order
        self._vflags = None
        self._attach_tgt = None
        self._pin_tgt = None
        self._attach_mats: list[tuple[float, float]] = []
        self._build_vertex_constraints()
        # parameters
        prm = capi.XpbdParams()
        prm.dt = float(dt)
        prm.gravity[:] = [float(x) for x in gravity_vec]
        prm.veldamping = float(veldamping)
        prm.quasi_static = int(bool(quasi_static))
        prm.omega = float(omega)
        prm.contraction_ratio = float(contraction_ratio)
        prm.fiber_stiffness_scale = float(fiber_stiffness_scale)
        prm.n_materials = len(L.materials)
        for i, m in enumerate(L.materials):
            for k, v in m.items():
                setattr(prm.materials[i], k, v)
        # fixed-point accumulation scale of the tile passes.  Its range must hold one
        # tet's corrections: a few edge lengths while the state is sane (the box
        # muscle's first sagging iterations reach 33 edges, 97 mm, summed over a
        # tet's 12 components), or a pin's jump between two poses, bounded by the
        # scene's extent.  Its quantum 1/acc_scale must stay well below the FP32
        # rounding of the corrections: corrections below half a quantum are lost,
        # a dead zone that an eighth as fine a scale showed on the 535k-tet
        # multigrid scene (stiff fibre tets at the tendon pins settled into a
        # different state).  Range = 64-128 longest rest edges or 0.5-1 x the
        # largest rest coordinate, whichever is larger: quantum 1.5e-8 m on the
        # 535k-tet scene, 7.5e-9 m on the box.
        e = getattr(self, "_acc_range", None)
        if e is None:
            e = max_rest_edge(self.pos0_np, self.tet_np) if self.tet_np.size else 0.0
            e = max(ACC_RANGE_EDGES * e, float(np.abs(self.pos0_np).max()))
        e = max(float(e), 1e-9)
        prm.acc_scale = float(self._lib.xpbd_acc_scale_for_extent(e))
        prm.status = self._pstatus.data_ptr()
        prm.n_attach_materials = len(self._attach_mats)
        for i, (k, d) in enumerate(self._attach_mats):
            prm.attach[i].k = k
            prm.attach[i].damp = d
        self._prm = prm
        self.dt = float(dt)
        self._sdf = None
        self._graphs: dict = {}
        self._refresh_structs()
        torch.cuda.synchronize(dev)

    def _inv_mass_user(self) -> np.ndarray:
        """get_inv_mass_fn (solve_kernels.py:71-80), folded into pos.w."""
        m = self._mass_user
        inv = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0).astype(np.float32)
        inv[self._stopped_user != 0] = 0.0
        return inv

    def _build_vertex_constraints(self) -> None:
        """ATTACH rows of the table -> per-vertex attach slots (library order)."""
        tb = self.table
        rng = tb.cons_ranges.get(ConstraintType.ATTACH)
        nv = self.n_verts
        L = self.layout
        flags = np.zeros(nv, np.int32)
        att = np.zeros((nv, 4), np.float32)
        if rng is not None:
            off, cnt = rng
            sl = slice(off, off + cnt)
            src = tb.c_pts[sl, 0]
            if np.unique(src).shape[0] != src.shape[0]:
                raise NotImplementedError("two ATTACH constraints on one vertex are not supported")
            keys = np.stack([tb.c_stiffness[sl], tb.c_dampingratio[sl]], 1)
            uk, mat_of = np.unique(keys, axis=0, return_inverse=True)
            if uk.shape[0] > capi.MAX_ATTACH_MATERIALS:
                raise ValueError("too many distinct ATTACH (stiffness, dampingratio) pairs")
            self._attach_mats = [(float(a), float(b)) for a, b in uk]
            flags[src] = mat_of.ravel().astype(np.int32) + 1
            att[src, :3] = tb.c_restvector[sl, :3]
            att[src, 3] = tb.c_restlength[sl]
            self._attach_row_of_vertex = np.full(nv, -1, np.int64)
            self._attach_row_of_vertex[src] = np.arange(off, off + cnt)
        pin = getattr(self, "_pin_user", None)  # (has_pin (nv,), target (nv,3), active (nv,)) from subclasses
        pin4 = np.zeros((nv, 4), np.float32)
        if pin is not None:
            has, tgt, act = pin
            flags |= np.where(np.asarray(has) != 0, capi.VF_PIN, 0).astype(np.int32)
            pin4[:, :3] = tgt
            pin4[:, 3] = (np.asarray(act) != 0)
        # the soft pin of all constraint points (presubframe_pintotarget) reads the
        # pin targets even where no vertex is pinned or attached
        if flags.any() or (pin is not None and float(getattr(self, "presubframe_pintotarget", 0.0)) > 0.0):
            dev = self.device
            self._vflags = torch.from_numpy(flags[L.perm]).to(dev)
            self._attach_tgt = torch.from_numpy(att[L.perm]).to(dev)
            self._pin_tgt = torch.from_numpy(pin4[L.perm]).to(dev)

    def _refresh_structs(self) -> None:
        v = capi.XpbdVerts()
        v.n = self.n_verts
        v.pos, v.pprev, v.vel = _ptr(self._pos4), _ptr(self._prev4), _ptr(self._vel4)
        v.mass, v.force, v.accum = _ptr(self._massd), None, _ptr(self._accum)
        v.vflags, v.attach_target, v.pin_target = _ptr(self._vflags), _ptr(self._attach_tgt), _ptr(self._pin_tgt)
        self._verts = v
        L = self.layout
        t = capi.XpbdTiles()
        t.n_tets, t.n_tiles, t.n_boundary, t.max_tile_verts = L.n_tets, L.n_tiles, L.n_boundary, L.max_tile_verts
        t.tile_vptr, t.tile_nint, t.tile_tptr = _ptr(self._t_vptr), _ptr(self._t_nint), _ptr(self._t_tptr)
        t.tile_verts, t.tet_q = _ptr(self._t_verts), _ptr(self._t_q)
        t.tet_b0, t.tet_b1, t.tet_b2 = _ptr(self._t_b0), _ptr(self._t_b1), _ptr(self._t_b2)
        t.tet_fiber, t.tet_act = _ptr(self._t_fiber), _ptr(self._t_act)
        t.bnd_verts = _ptr(self._t_bnd)
        t.vert_ntiles, t.arrive = _ptr(self._t_ntiles), _ptr(self._t_arrive)
        self._tiles = t
        # orphan vertices (in no tet) still take ATTACH/pin in the fused pass
        to = capi.XpbdTiles()
        C.memmove(C.addressof(to), C.addressof(t), C.sizeof(t))
        if self._t_orph is not None:
            to.n_boundary, to.bnd_verts = int(self._t_orph.shape[0]), _ptr(self._t_orph)
        else:
            to.n_boundary = 0
        self._tiles_orph = to
        fits, slots = C.c_int32(0), C.c_int32(0)
        capi.check(self._lib.xpbd_persistent_fits(C.byref(self._prm), C.byref(t), C.byref(fits), C.byref(slots)))
        self._persist_slots = int(slots.value)
        self._build_persist(self._persist_slots)
        for g in self._graphs.values():
            capi.check(self._lib.xpbd_graph_destroy(g))
        self._graphs = {}

    #: synchronisation between the iterations of the persistent pass: "grid"
    #: (one grid-wide barrier) or "neighbour" (each tile waits for the tiles it
    #: shares boundary vertices with)
    persistent_sync = "grid"

    def _tile_neighbours(self):
        """CSR of the tiles each tile shares a boundary vertex with (itself excluded)."""
        import scipy.sparse as sp
        L = self.layout
        nt = L.n_tiles
        counts = np.diff(L.tile_vptr)
        tile_of = np.repeat(np.arange(nt), counts)
        local = np.arange(L.tile_verts.shape[0]) - np.repeat(L.tile_vptr[:-1], counts)
        bnd = local >= np.repeat(L.tile_nint, counts)
        M = sp.csr_matrix((np.ones(int(bnd.sum()), np.int8), (tile_of[bnd], L.tile_verts[bnd])),
                          shape=(nt, L.n_verts))
        A = (M @ M.T).tocsr()
        A.setdiag(0)
        A.eliminate_zeros()
        A.sort_indices()
        return A.indptr.astype(np.int32), A.indices.astype(np.int32)

    def _build_persist(self, slots: int) -> None:
        """Persistent-pass launch descriptors for tile ranges of at most
        ``slots`` tiles (one set of barrier words per range)."""
        ranges = self._persist_ranges(int(slots))
        if 4 * len(ranges) > self._psync.numel():
            self._psync = torch.zeros(4 * len(ranges), dtype=torch.int32, device=self.device)
        ptr, idx = self._tile_neighbours()
        self._t_nbr_ptr = torch.from_numpy(ptr).to(self.device)
        self._t_nbr_idx = torch.from_numpy(idx if idx.size else np.zeros(1, np.int32)).to(self.device)
        self._t_cnt = torch.zeros(self.layout.n_tiles, dtype=torch.int32, device=self.device)
        # a vertex's ring slots follow its range's phase word: start all over
        with torch.cuda.stream(self._stream):
            self._ring.zero_()
            self._psync.zero_()
        self._stream.synchronize()
        self._persist = []
        nb = self.persistent_sync == "neighbour"
        for k, (b, e) in enumerate(ranges):
            ps = capi.XpbdPersist()
            ps.tile_own, ps.ring, ps.status = _ptr(self._t_own), _ptr(self._ring), _ptr(self._pstatus)
            ps.sync = self._psync.data_ptr() + 16 * k
            ps.tile_begin, ps.tile_end = b, e
            if nb:
                ps.nbr_ptr, ps.nbr_idx, ps.tile_cnt = (_ptr(self._t_nbr_ptr), _ptr(self._t_nbr_idx),
                                                       _ptr(self._t_cnt))
            self._persist.append(ps)
        self._persist_fits = bool(ranges)

    # -------------------------------------------------------------- launches
    def _vstep(self, ops: int) -> None:
        sdf = self._sdf.struct() if (ops & capi.OP_SDF) and self._sdf is not None else None
        if ops & capi.OP_SDF and sdf is None:
            ops &= ~capi.OP_SDF
        capi.check(self._lib.xpbd_vertex_step(C.byref(self._prm), C.byref(self._verts), ops,
                                              C.byref(sdf) if sdf is not None else None, self._sp))

    def _project(self, mode: int) -> None:
        capi.check(self._lib.xpbd_project(C.byref(self._prm), C.byref(self._tiles), C.byref(self._verts), mode,
                                          self._sp))

    def _apply_boundary(self, ops: int) -> None:
        capi.check(self._lib.xpbd_apply_boundary(C.byref(self._prm), C.byref(self._tiles), C.byref(self._verts), ops,
                                                 self._sp))

    def _apply_all(self, ops: int) -> None:
        capi.check(self._lib.xpbd_apply_all(C.byref(self._prm), C.byref(self._verts), ops, self._sp))

    def _fused_iteration(self) -> None:
        """clear -> solve_constraints -> apply_dP -> apply_pintotarget, fused.
        The fused pass expects an all-zero accumulator (it clears the slots it
        uses); a preceding unfused solve may have left sums behind."""
        if self._accum_dirty:
            self.clear()
        if self.fused_mode == capi.PROJECT_FUSED_LAST:
            self._project(capi.PROJECT_FUSED_LAST)
            if self._t_orph is not None and self._vflags is not None:
                capi.check(self._lib.xpbd_apply_boundary(C.byref(self._prm), C.byref(self._tiles_orph),
                                                         C.byref(self._verts),
                                                         capi.APPLY_ATTACH | capi.APPLY_DIVIDE | capi.APPLY_PIN
                                                         | capi.APPLY_CLEAR, self._sp))
            return
        self._project(capi.PROJECT_FUSED)
        self._apply_boundary(capi.APPLY_ATTACH | capi.APPLY_DIVIDE | capi.APPLY_PIN | capi.APPLY_CLEAR)

    def _persist_ranges(self, slots: int) -> list[tuple[int, int]]:
        """Tile ranges of the persistent pass: all tiles when they fit in the
        resident CTA slots; for a layout of independent vertex groups, runs of
        whole groups of at most ``slots`` tiles each; [] when neither works."""
        L = self.layout
        if slots <= 0:
            return []
        if L.n_tiles <= slots:
            return [(0, L.n_tiles)]
        if L.tile_group is None:
            return []
        starts = np.r_[0, np.nonzero(np.diff(L.tile_group))[0] + 1, L.n_tiles]
        ranges, b = [], 0
        for e0, e1 in zip(starts[:-1], starts[1:]):
            if e1 - e0 > slots:
                return []
            if e1 - b > slots:
                ranges.append((b, int(e0)))
                b = int(e0)
        ranges.append((b, L.n_tiles))
        return ranges

    def _fused_iterations(self, n: int) -> None:
        """n fused iterations: one persistent cooperative launch per tile range
        when the tiles fit on the GPU at once, else n x _fused_iteration()."""
        if n <= 0:
            return
        if self.use_persistent and self._persist_fits and self.fused_mode == capi.PROJECT_FUSED:
            for ps in self._persist:
                capi.check(self._lib.xpbd_iterate_persistent(C.byref(self._prm), C.byref(self._tiles),
                                                             C.byref(self._verts), C.byref(ps), int(n), self._sp))
            return
        for _ in range(n):
            self._fused_iteration()

    def persistent_status(self, reset: bool = True) -> int:
        """XPBD_STATUS_* bits of the persistent pass and of the tile passes'
        fixed-point range check (synchronises).  After a barrier timeout the
        ring and barrier words are cleared for the next launch."""
        self._stream.synchronize()
        st = int(self._pstatus.item())
        self._status_pending = False  # this read supersedes the copy queued behind the last frame
        if st and reset:
            with torch.cuda.stream(self._stream):
                self._ring.zero_()
                self._psync.zero_()
                self._t_cnt.zero_()
                self._pstatus.zero_()
            self._stream.synchronize()
        return st

    def _post_status(self) -> None:
        """Queue copies of the device status words (the tile passes' word and,
        with a DCD attached, the DCD's) into pinned host memory behind the
        work launched so far, with an event; no synchronisation."""
        with torch.cuda.stream(self._stream):
            self._status_host[0:1].copy_(self._pstatus, non_blocking=True)
            dcd = getattr(self, "dcd", None)
            if dcd is not None:
                self._status_host[1:2].copy_(dcd.buf.t["counters"][2:3], non_blocking=True)
        if self._status_event is None:
            self._status_event = torch.cuda.Event()
        self._status_event.record(self._stream)
        self._status_pending = True

    def _check_status(self) -> None:
        """Raise if the last status copy that has landed shows a fatal bit.

        A barrier timeout leaves the persistent pass's later barriers giving
        up early (the bit is sticky), and a fixed-point range overflow
        wraps the sums: both make every later result wrong without any other
        sign.  Called before each frame (non-blocking: a copy still in flight
        is checked at the next call) and after every synchronising read.
        Before raising, the barrier words, ring, status word and the DCD's
        counters are cleared, so the next launch runs with full barriers."""
        if not getattr(self, "_status_pending", False) or not self._status_event.query():
            return
        self._status_pending = False
        st, sd = (int(x) for x in self._status_host.tolist())
        msg = status_error(st, sd if getattr(self, "dcd", None) is not None else 0)
        if msg is None:
            return
        with torch.cuda.stream(self._stream):
            self._ring.zero_()
            self._psync.zero_()
            self._t_cnt.zero_()
            self._pstatus.zero_()
            dcd = getattr(self, "dcd", None)
            if dcd is not None:
                dcd.buf.reset()
        self._stream.synchronize()
        raise RuntimeError(msg)

    def synchronize(self) -> None:
        self._stream.synchronize()
        self._check_status()

    # ------------------------------------------- reference engine primitives
    def integrate(self) -> None:
        """XpbdEngine.integrate (engine.py:798-809)."""
        self._vstep(capi.OP_PREDICT)

    def update_velocities(self) -> None:
        """XpbdEngine.update_velocities (engine.py:811-829); no-op when quasi-static."""
        if self._prm.quasi_static:
            return
        self._vstep(capi.OP_VELOCITY)

    def clear(self) -> None:
        """XpbdEngine.clear (engine.py:858-863): zero dP/dPw (c_L is identically 0 on the Jacobi path)."""
        with torch.cuda.stream(self._stream):
            self._accum.zero_()
        self._accum_dirty = False

    def solve_constraints(self, run_extras: bool = True) -> None:
        """XpbdEngine.solve_constraints (engine.py:1029-1052): accumulate every constraint into dP/dPw."""
        extras = getattr(self, "constraint_solvers", None)
        if self.n_cons > 0:
            self._accum_dirty = True
            self._project(capi.PROJECT_ACCUMULATE)
            if self._vflags is not None:
                self._apply_all(capi.APPLY_ATTACH)
        if run_extras and extras:
            for fn in extras:
                fn()

    def solve_extras(self) -> None:
        """XpbdEngine.solve_extras (engine.py:1054-1067)."""
        for fn in getattr(self, "constraint_solvers", None) or []:
            fn()

    def apply_dP(self) -> None:
        """XpbdEngine.apply_dP (engine.py:865-867)."""
        self._apply_all(capi.APPLY_DIVIDE)

    def apply_pintotarget(self) -> None:
        """Hard pin of the per-vertex pin targets (mg/mg.py:1251-1261)."""
        if self._vflags is not None and getattr(self, "_has_pins", False):
            self._apply_all(capi.APPLY_PIN)

    def post_smooth(self) -> None:
        """XpbdEngine.post_smooth (engine.py:1072-1100): extra Jacobi sweeps of the
        non-fiber constraints (every type on this path)."""
        n = int(self._option("post_smooth_iters", 0))
        for _ in range(n):
            self.clear()
            self.solve_constraints(run_extras=False)
            self.apply_dP()
            self.apply_pintotarget()

    def freeze_near_inverted(self) -> None:
        """XpbdEngine.freeze_near_inverted (engine.py:1102-1124): disabled on CUDA
        devices in the reference (races on shared vertices); same here."""
        if float(self._option("freeze_detF_threshold", 0.0)) > 0.0 and not getattr(self, "_freeze_warned", False):
            log.warning("freeze_near_inverted skipped on GPU (race condition on shared vertices)")
            self._freeze_warned = True

    def _option(self, name: str, default):
        """An engine option: an attribute of the engine, else of its config (a
        dict or the reference's SimConfig object)."""
        if hasattr(self, name):
            return getattr(self, name)
        cfg = getattr(self, "cfg", None)
        if isinstance(cfg, dict):
            return cfg.get(name, default)
        return getattr(cfg, name, default)

    def repair_inverted_tets(self) -> None:
        """XpbdEngine.repair_inverted_tets (engine.py:831-856): repair_iters
        passes of the SVD clamp (singular values raised to repair_sigma_min,
        Jacobi-averaged, blended by repair_alpha); off unless repair_alpha > 0
        and repair_iters > 0."""
        alpha = float(self._option("repair_alpha", 0.0))
        iters = int(self._option("repair_iters", 0))
        if alpha <= 0.0 or iters <= 0:
            return
        sigma_min = float(self._option("repair_sigma_min", 0.1))
        capi.check(self._lib.xpbd_svd_clamp(C.byref(self._tiles), C.byref(self._verts), C.c_float(sigma_min),
                                            C.c_float(alpha), iters, self._sp))
        self._accum_dirty = False  # the clamp leaves the accumulator zeroed

    def run_program(self) -> None:
        """XpbdEngine.run_program (engine.py:1126-1134)."""
        for sub in range(self.num_substeps):
            self._program_sub = sub
            for phase in self.program:
                phase()

    # ------------------------------------------------------------- metrics
    def metrics(self) -> dict:
        out = self._metrics_buf
        capi.check(self._lib.xpbd_metrics(C.byref(self._tiles), C.byref(self._verts), C.c_void_p(out.data_ptr()),
                                          self._sp))
        self._stream.synchronize()
        raw = out.cpu().numpy().tobytes()
        m = capi.XpbdMetrics.from_buffer_copy(raw[:C.sizeof(capi.XpbdMetrics)])
        return dict(vol_sum=m.vol_sum, resid_sq_sum=m.resid_sq_sum, resid_max=m.resid_max, n_inverted=m.n_inverted,
                    n_nonfinite=m.n_nonfinite)

    def count_inverted(self) -> int:
        """MuscleSim.count_inverted (musclesim.py:669-675)."""
        return int(self.metrics()["n_inverted"])

    def calc_vol_error(self) -> float:
        """MuscleSim.calc_vol_error (musclesim.py:658-667)."""
        tot = float(self.total_rest_volume)
        if tot == 0.0:
            return 0.0
        return (self.metrics()["vol_sum"] - tot) / tot

    # ------------------------------------------------------ user-order views
    def _to_user(self, t4: torch.Tensor, ncol: int = 3) -> np.ndarray:
        self.synchronize()
        a = t4[:, :ncol].cpu().numpy()
        out = np.empty_like(a)
        out[self.layout.perm] = a
        return out

    def positions_np(self) -> np.ndarray:
        return self._to_user(self._pos4)

    @property
    def pos(self) -> torch.Tensor:
        """Current positions (NV,3) in the user's vertex order (a copy)."""
        return torch.from_numpy(self.positions_np())

    @property
    def pprev(self) -> torch.Tensor:
        return torch.from_numpy(self._to_user(self._prev4))

    @property
    def vel(self) -> torch.Tensor:
        return torch.from_numpy(self._to_user(self._vel4))

    @property
    def dP(self) -> torch.Tensor:
        return torch.from_numpy(self._to_user(self._accum))

    @property
    def dPw(self) -> torch.Tensor:
        return torch.from_numpy(self._to_user(self._accum, 4)[:, 3].copy())

    def __getattr__(self, name: str):
        """The constraint table's columns as the reference engine's ``c_*``
        attributes (engine.py:1179-1211: c_type, c_pts, c_stiffness,
        c_compressionstiffness, c_dampingratio, c_tetid, c_L, c_restlength,
        c_restvector, c_restdir), type-sorted rows with user vertex ids, as
        device tensors.  They are copies of the table the engine was built
        from: writing to them changes nothing (rebuild_constraints does)."""
        table = self.__dict__.get("table")
        if name.startswith("c_") and table is not None and name in table.__dataclass_fields__:
            return torch.from_numpy(np.ascontiguousarray(getattr(table, name))).to(self.device)
        raise AttributeError(f"{type(self).__name__!r} object has no attribute {name!r}")

    @property
    def mass(self) -> np.ndarray:
        return self._mass_user.copy()

    @property
    def stopped(self) -> np.ndarray:
        return self._stopped_user.copy()

    @stopped.setter
    def stopped(self, value) -> None:
        """Set the per-vertex 'stopped' flags (kinematic, inverse mass 0)."""
        if isinstance(value, torch.Tensor):
            value = value.detach().cpu().numpy()
        self._stopped_user = np.asarray(value, np.int32).reshape(self.n_verts).copy()
        self._upload_w_lanes()

    def _upload_w_lanes(self) -> None:
        perm = self.layout.perm
        inv = torch.from_numpy(self._inv_mass_user()[perm]).to(self.device)
        stp = torch.from_numpy((self._stopped_user[perm] != 0).astype(np.float32)).to(self.device)
        with torch.cuda.stream(self._stream):
            self._pos4[:, 3] = inv
            self._vel4[:, 3] = stp
        self._stream.synchronize()

    def set_positions(self, pos_np: np.ndarray, also_prev: bool = False) -> None:
        p = np.asarray(pos_np, np.float32)[self.layout.perm]
        t = torch.from_numpy(p).to(self.device)
        with torch.cuda.stream(self._stream):
            self._pos4[:, :3] = t
            if also_prev:
                self._prev4[:, :3] = t
        self._stream.synchronize()

    def set_velocities(self, vel_np: np.ndarray) -> None:
        v = torch.from_numpy(np.asarray(vel_np, np.float32)[self.layout.perm]).to(self.device)
        with torch.cuda.stream(self._stream):
            self._vel4[:, :3] = v
        self._stream.synchronize()

    # --------------------------------------------------------------- graphs
    def _graph(self, key, body) -> None:
        """Capture ``body`` (a sequence of library launches on the engine stream)
        once per key, then replay it."""
        if not self.use_graphs:
            body()
            return
        g = self._graphs.get(key)
        if g is None:
            capi.check(self._lib.xpbd_graph_begin(self._sp))
            try:
                body()
            except Exception:
                ex = C.c_void_p()
                self._lib.xpbd_graph_end(self._sp, C.byref(ex))
                if ex.value:
                    self._lib.xpbd_graph_destroy(ex)
                raise
            ex = C.c_void_p()
            capi.check(self._lib.xpbd_graph_end(self._sp, C.byref(ex)))
            g = self._graphs[key] = ex
        capi.check(self._lib.xpbd_graph_launch(g, self._sp))

    def release_graphs(self) -> None:
        for g in self._graphs.values():
            self._lib.xpbd_graph_destroy(g)
        self._graphs = {}

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:
            pass


class XpbdSolver(XpbdEngine):
    """The engine over explicit arrays: a mesh plus a reference-layout constraint
    table (the plugin-level entry used by tests, batching and tools)."""

    def __init__(self, verts, tets, table: ConstraintTable, *, mass, dt, stopped=None, gravity=(0.0, 0.0, 0.0),
                 veldamping=0.0, quasi_static=False, relaxation=1.0, v_fiber=None, tet_tendonmask=None,
                 contraction_ratio=0.0, fiber_stiffness_scale=1.0, device="cuda:0", tile_tets=None, pins=None,
                 num_substeps=1, total_rest_volume=None, stream=None, acc_range=None):
        """``acc_range``: the length the fixed-point accumulator's per-tet range is
        sized for (default: the larger of 128 longest rest edges and the largest
        rest coordinate)."""
        self._acc_range = acc_range
        self.pos0_np = np.asarray(verts, np.float32)
        self.tet_np = np.asarray(tets, np.int32)
        self.n_verts = self.pos0_np.shape[0]
        self.num_substeps = int(num_substeps)
        self.quasi_static = bool(quasi_static)
        if pins is not None:
            self._pin_user = pins
            self._has_pins = True
        if total_rest_volume is None:
            from .builder import lumped_mass
            total_rest_volume = float(lumped_mass(self.pos0_np, self.tet_np, 1.0)[1].astype(np.float64).sum())
        self.total_rest_volume = total_rest_volume
        st = np.zeros(self.n_verts, np.int32) if stopped is None else stopped
        self._setup_device(device, mass=mass, stopped=st, table=table, v_fiber=v_fiber,
                           tet_tendonmask=tet_tendonmask, dt=dt, gravity_vec=gravity, veldamping=veldamping,
                           quasi_static=quasi_static, omega=relaxation, contraction_ratio=contraction_ratio,
                           fiber_stiffness_scale=fiber_stiffness_scale, tile_tets=tile_tets, stream=stream)

    def project_once(self) -> None:
        """clear -> solve_constraints -> apply_dP -> apply_pintotarget (unfused primitives)."""
        self.clear()
        self.solve_constraints(run_extras=False)
        self.apply_dP()
        self.apply_pintotarget()

    def iterate_fused(self) -> None:
        self._fused_iteration()

    def set_activation(self, acti_np) -> None:
        a = np.ascontiguousarray(np.asarray(acti_np, np.float32)[self.layout.tet_perm])
        with torch.cuda.stream(self._stream):
            self._t_act.copy_(torch.from_numpy(a).to(self.device))
        self._stream.synchronize()
