"""MuscleSim on the sm_100a engine (reference: src/muscle/musclesim.py).

``MuscleSim.from_procedural`` (musclesim.py:181-287) is the no-asset entry
point; ``MuscleSim(cfg)`` (musclesim.py:44-92) reads the rest mesh from a
Houdini ``.geo`` file or a text USD layer (``.usda``, read without pxr) at
``cfg.geo_path``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import torch

from . import _capi as capi

from .builder import ConstraintTable, collect_raw_constraints, create_attach_constraints, lumped_mass
from .engine import XpbdEngine


class _GeoPointAttrs:
    """Point attributes of a .geo rest mesh as attributes (the reference's
    ``self.geo``, read by the attach blocks' ``mask_name``)."""

    def __init__(self, geo):
        self._geo = geo

    def __getattr__(self, name):
        geo = self.__dict__["_geo"]
        if geo.has_point_attr(name):
            return geo.point_attr(name)
        raise AttributeError(name)


class MuscleSim(XpbdEngine):
    """XPBD muscle simulator: one Jacobi projection per substep."""

    def __init__(self, cfg, device: str = "cuda:0"):
        """MuscleSim(cfg) (musclesim.py:44-92): the rest mesh from ``cfg.geo_path``
        (a Houdini ``.geo`` tet mesh, geo.scene_from_geo, or the TetMesh of a text
        USD layer, usd.scene_from_usda, with ``cfg.geo_prim_path`` choosing the
        prim: points, tets, the ``materialW`` fiber field and ``tendonmask``), the constraint blocks of
        ``cfg.constraints``, ``dt`` / ``num_substeps``, ``density``,
        ``veldamping``, ``gravity`` (along Y), ``contraction_ratio``,
        ``fiber_stiffness_scale``.  ``cfg`` is a dict or an attribute object
        (the reference's SimConfig)."""
        get = (lambda k, d=None: cfg.get(k, d)) if isinstance(cfg, dict) else (lambda k, d=None: getattr(cfg, k, d))
        # musclesim.py:73-74: use_jacobi (default true on a GPU) and use_colored_gs;
        # the Gauss-Seidel solves are refused rather than silently replaced
        if not bool(get("use_jacobi", True)) or bool(get("use_colored_gs", False)):
            raise NotImplementedError("use_jacobi=false / use_colored_gs=true select the reference's Gauss-Seidel "
                                      "solves, which are not on the sm_100a path (it runs the Jacobi projection)")
        path = get("geo_path")
        if not path:
            raise ValueError("MuscleSim(cfg) needs cfg.geo_path (or use MuscleSim.from_procedural)")
        path = Path(path)
        if path.suffix.lower() not in (".geo", ".usda", ".usd"):
            raise NotImplementedError(f"{path.name}: rest meshes are read from Houdini .geo files and text USD "
                                      "layers (.usda)")
        if not path.exists():
            raise FileNotFoundError(f"geo_path {path} does not exist")
        if path.suffix.lower() == ".geo":
            from .geo import GeoFile, scene_from_geo
            sc = scene_from_geo(path)
            self.geo = _GeoPointAttrs(GeoFile(path))
        else:
            from .usd import scene_from_usda
            sc = scene_from_usda(path, get("geo_prim_path"))
            self.geo = SimpleNamespace(tendonmask=sc.v_tendon)
        self.bone_pos = np.zeros((0, 3), np.float32)
        tendon_tet = (sc.v_tendon[sc.tets].astype(np.float32).sum(1) / np.float32(4.0)).astype(np.float32)
        self._build(sc.verts, sc.tets, sc.v_fiber, cfg=cfg, constraint_configs=list(get("constraints") or []),
                    dts=float(get("dt", 1.0 / 24.0)), num_substeps=int(get("num_substeps", 1)), device=device,
                    density=float(get("density", 1060.0)), veldamping=float(get("veldamping", 0.02)),
                    gravity=float(get("gravity", 0.0)), contraction_ratio=float(get("contraction_ratio", 0.4)),
                    fiber_stiffness_scale=float(get("fiber_stiffness_scale", 10000.0)),
                    quasi_static=bool(get("quasi_static", False)), tet_tendonmask=tendon_tet,
                    v_tendonmask=sc.v_tendon)

    @classmethod
    def from_procedural(cls, vertices, tets, fiber_dirs_per_tet, bone_targets=None, *, constraint_configs, dts,
                        num_substeps=1, device="cuda:0", density=1060.0, veldamping=0.02, gravity=0.0, sigma0=0.0,
                        lambda_opt=1.0, contraction_ratio=0.0, fiber_stiffness_scale=1.0, v_max_norm=0.0,
                        d_damp=0.0, stopped=None, relaxation=1.0, tile_tets=None, tet_masks=None):
        """Build a MuscleSim from mesh arrays (musclesim.py:181-287).

        Extra keywords beyond the reference: ``stopped`` (per-vertex kinematic
        flags, equivalent to assigning ``sim.stopped`` afterwards),
        ``relaxation`` (scale of the averaged Jacobi correction; 1 reproduces
        the reference's apply_dP), ``tile_tets`` (tile size of the tet pass)
        and ``tet_masks`` (restrict a named constraint config to a tet subset).
        """
        if float(sigma0) > 0.0:
            raise NotImplementedError("explicit active fiber force (sigma0 > 0) is not on the sm_100a path")
        vertices = np.asarray(vertices, dtype=np.float32)
        tets = np.asarray(tets, dtype=np.int32)
        n_v = vertices.shape[0]
        fd = np.asarray(fiber_dirs_per_tet, dtype=np.float32).reshape(-1, 3)
        # per-tet -> per-vertex fiber average (musclesim.py:226-234)
        vf = np.zeros((n_v, 3), dtype=np.float32)
        vc = np.zeros(n_v, dtype=np.float32)
        np.add.at(vf, tets.reshape(-1), np.repeat(fd, 4, axis=0))
        np.add.at(vc, tets.reshape(-1), np.float32(1.0))
        vc = np.maximum(vc, np.float32(1.0))
        vf /= vc[:, None]
        vf /= np.maximum(np.linalg.norm(vf, axis=1, keepdims=True), np.float32(1e-8))
        cfg = SimpleNamespace(
            geo_path="<procedural>", bone_geo_path="<none>", gui=False, render_mode="none",
            constraints=list(constraint_configs), dt=dts, num_substeps=num_substeps, gravity=gravity,
            density=density, veldamping=veldamping, contraction_ratio=contraction_ratio,
            fiber_stiffness_scale=fiber_stiffness_scale, HAS_compressstiffness=False, arch=device,
            activation=0.0, nsteps=1, sigma0=sigma0, lambda_opt=lambda_opt, v_max_norm=v_max_norm, d_damp=d_damp,
            relaxation=relaxation)
        sim = object.__new__(cls)
        sim.geo = SimpleNamespace()  # point attributes for attach masks, as the reference's empty namespace
        sim._build(vertices, tets, vf, cfg=cfg, constraint_configs=cfg.constraints, dts=dts,
                   num_substeps=num_substeps, device=device, density=density, veldamping=veldamping, gravity=gravity,
                   contraction_ratio=contraction_ratio, fiber_stiffness_scale=fiber_stiffness_scale, stopped=stopped,
                   relaxation=relaxation, tile_tets=tile_tets, tet_masks=tet_masks, bone_targets=bone_targets)
        return sim

    def _build(self, vertices, tets, v_fiber, *, cfg, constraint_configs, dts, num_substeps, device, density,
               veldamping, gravity, contraction_ratio, fiber_stiffness_scale, stopped=None, relaxation=1.0,
               tile_tets=None, tet_masks=None, bone_targets=None, quasi_static=False, tet_tendonmask=None,
               v_tendonmask=None) -> None:
        """Common set-up of both constructors: constraint table, lumped mass,
        device state."""
        vertices = np.asarray(vertices, dtype=np.float32)
        tets = np.asarray(tets, dtype=np.int32)
        n_v = vertices.shape[0]
        self.cfg = cfg
        self.constraint_configs = list(constraint_configs)
        self.pos0_np = vertices
        self.tet_np = tets
        self.v_fiber_np = np.asarray(v_fiber, np.float32)
        self.v_tendonmask_np = v_tendonmask
        self.n_verts = n_v
        if bone_targets is not None:
            self.bone_pos = np.asarray(bone_targets, np.float32).reshape(-1, 3)
        elif not hasattr(self, "bone_pos"):
            self.bone_pos = np.zeros((0, 3), np.float32)
        if not hasattr(self, "geo"):
            self.geo = SimpleNamespace()
        self.use_jacobi = True
        self.use_colored_gs = False
        self.contraction_ratio = contraction_ratio
        self.fiber_stiffness_scale = fiber_stiffness_scale
        self.has_compressstiffness = False
        self.num_substeps = int(num_substeps)
        self.quasi_static = bool(quasi_static)
        self.step_cnt = 0
        self.renderer = None
        mass, rest_volume = lumped_mass(vertices, tets, density)
        self.rest_volume_np = rest_volume
        self.total_rest_volume = float(rest_volume.astype(np.float64).sum())
        self._tet_masks = tet_masks
        table = collect_raw_constraints(vertices, tets, self.constraint_configs, tet_masks)
        attach = self._bone_attach_rows(vertices, tets)
        if attach is not None:
            table = ConstraintTable.concat([table, attach])
        table = table.sorted_by_type()
        self.raw_constraints = table
        st = np.zeros(n_v, np.int32) if stopped is None else np.asarray(stopped, np.int32)
        self._setup_kw = dict(device=device, mass=mass, v_fiber=self.v_fiber_np, tet_tendonmask=tet_tendonmask,
                              dt=float(dts) / int(num_substeps), gravity_vec=(0.0, float(gravity), 0.0),
                              veldamping=float(veldamping), quasi_static=bool(quasi_static),
                              omega=float(relaxation), contraction_ratio=contraction_ratio,
                              fiber_stiffness_scale=fiber_stiffness_scale, tile_tets=tile_tets)
        self._setup_device(stopped=st, table=table, **self._setup_kw)

    # ------------------------------------------------------- state helpers
    def reset(self) -> None:
        """reset (musclesim.py:555-562): rest positions (also the previous ones),
        zero velocities and activation, cleared accumulators, step count 1."""
        self.set_positions(self.pos0_np, also_prev=True)
        self.set_velocities(np.zeros_like(self.pos0_np))
        if self._t_act is not None:
            with torch.cuda.stream(self._stream):
                self._t_act.zero_()
        self.clear()
        self.synchronize()
        self.step_cnt = 1

    def clear_forces(self) -> None:
        """clear_forces (musclesim.py:580-582).  The explicit per-vertex force
        accumulator only feeds the active fiber force (sigma0 > 0), which this
        path does not run, so there is nothing to zero."""

    def clear_reaction(self) -> None:
        """clear_reaction (musclesim.py:676-679).  The attach reaction sums are
        not accumulated on this path (get_insertion_force works from
        positions), so there is nothing to zero."""

    def save_predicted_positions(self, vertex_ids) -> None:
        """save_predicted_positions (musclesim.py:612-615): the positions of
        vertex_ids after integrate(), before the constraint solve."""
        ids = np.asarray(vertex_ids)
        self._predicted_pos = self.positions_np()[ids].copy()
        self._predicted_ids = ids

    def get_insertion_force(self, insertion_vids, dts) -> np.ndarray:
        """get_insertion_force (musclesim.py:617-633): net force on the bone,
        -sum m (x_corrected - x_predicted) / dts^2 over the insertion vertices
        (save_predicted_positions must have run after integrate())."""
        ids = np.asarray(insertion_vids)
        corrected = self.positions_np()[ids].astype(np.float64)
        masses = self._mass_user[ids].astype(np.float64)
        forces = masses[:, None] * (corrected - self._predicted_pos.astype(np.float64)) / (float(dts) * float(dts))
        return (-forces.sum(axis=0)).astype(np.float32)

    def set_lbs_T_rel(self, T_rel_flat_np) -> None:
        """set_lbs_T_rel (musclesim.py:635-644): per-bone relative transforms,
        (n_bones * 12,) row-major in the reference's row-vector layout
        [r00..r22, t0..t2] (q = p R + t), kept on the device as 3x4 [R^T | t]."""
        T = np.asarray(T_rel_flat_np, np.float32).reshape(-1, 12)
        M = np.concatenate([T[:, [0, 3, 6, 9]], T[:, [1, 4, 7, 10]], T[:, [2, 5, 8, 11]]], axis=1)
        self._lbs_T = torch.from_numpy(np.ascontiguousarray(M)).to(self.device)

    def apply_lbs(self, vertex_bone_field, blend: float = 1.0) -> None:
        """apply_lbs (musclesim.py:646-656; lbs_apply_kernel, engine.py:641-661):
        pos moves by ``blend`` toward its rest position carried by its bone's
        T_rel (vertices with bone < 0 stay).  Two device launches: the targets
        (xpbd_bone_targets) and the blend (xpbd_blend_to_target)."""
        T = getattr(self, "_lbs_T", None)
        if T is None:
            return
        vb = vertex_bone_field
        if isinstance(vb, torch.Tensor):
            vb = vb.detach().cpu().numpy()
        vb = np.asarray(vb, np.int32).reshape(self.n_verts)[self.layout.perm]
        vb2 = torch.from_numpy(np.ascontiguousarray(np.stack([vb, vb], 1))).to(self.device)
        if getattr(self, "_rest4_lbs", None) is None:
            r4 = np.zeros((self.n_verts, 4), np.float32)
            r4[:, :3] = self.pos0_np
            self._rest4_lbs = torch.from_numpy(r4[self.layout.perm]).to(self.device)
        with torch.cuda.stream(self._stream):
            tgt = self._pos4.clone()  # vertices without a bone blend toward themselves
        capi.check(self._lib.xpbd_bone_targets(self.n_verts, int(T.shape[0]), C.c_void_p(T.data_ptr()),
                                               C.c_void_p(vb2.data_ptr()), None, C.c_void_p(self._rest4_lbs.data_ptr()),
                                               C.c_void_p(tgt.data_ptr()), None, self._sp))
        capi.check(self._lib.xpbd_blend_to_target(self.n_verts, None, self.n_verts, C.c_void_p(self._pos4.data_ptr()),
                                                  C.c_void_p(tgt.data_ptr()), C.c_float(blend), self._sp))
        self.synchronize()

    # ------------------------------------------------------- bone attach
    def load_bone_geo(self, target_path):
        """load_bone_geo (musclesim.py:101-105): the bone geometry of an attach
        block (a Houdini .geo) and its point positions, read once."""
        if getattr(self, "_bone_geo_path", None) != str(target_path) or self.bone_pos.shape[0] == 0:
            from .geo import GeoFile
            self.bone_geo = GeoFile(target_path)
            self.bone_pos = self.bone_geo.positions.astype(np.float32)
            self._bone_geo_path = str(target_path)
        return getattr(self, "bone_geo", None), self.bone_pos

    def _bone_attach_rows(self, pos0, tets):
        """create_attach_constraints (builder.py:347-398) for every enabled
        "attach" block: the vertices whose point attribute ``mask_name`` exceeds
        ``mask_threshold`` (0.75) attach to their nearest bone point (a k-d tree
        over the bone points, from ``bone_targets`` or the block's
        ``target_path``) with the rest length of that distance.  Bone point
        groups (target_group) are not read: every bone point is a candidate."""
        from scipy.spatial import cKDTree
        rows = []
        self._attach_src = np.zeros(0, np.int64)
        self._attach_tgt_idx = np.zeros(0, np.int64)
        for params in self.constraint_configs:
            if not params.get("enable", True) or str(params.get("type", "")).lower() != "attach":
                continue
            if params.get("target_path") and self.bone_pos.shape[0] == 0:
                self.load_bone_geo(params["target_path"])
            mask = getattr(self.geo, str(params.get("mask_name")), None)
            if mask is None or self.bone_pos.shape[0] == 0:
                continue  # the reference warns and builds no rows
            src = np.nonzero(np.asarray(mask, np.float32).reshape(-1) > float(params.get("mask_threshold", 0.75)))[0]
            if src.size == 0:
                continue
            d, tgt = cKDTree(self.bone_pos).query(pos0[src], k=1)
            tgt = np.asarray(tgt, np.int64)
            first_tet = np.full(pos0.shape[0], -1, np.int64)
            order = np.arange(tets.shape[0] * 4)[::-1]
            first_tet[tets.reshape(-1)[order]] = order // 4
            rows.append(create_attach_constraints(
                src.astype(np.int32), self.bone_pos[tgt], np.asarray(d, np.float32),
                float(params.get("stiffness", 1e10)), float(params.get("dampingratio", 0.0)),
                tgt_idx=tgt.astype(np.int32), tetid=first_tet[src]))
            self._attach_src = np.concatenate([self._attach_src, src])
            self._attach_tgt_idx = np.concatenate([self._attach_tgt_idx, tgt])
        return ConstraintTable.concat(rows) if rows else None

    def update_attach_targets(self) -> None:
        """update_attach_targets (musclesim.py:564-578): the bone-attach targets
        follow the current bone points (``self.bone_pos``); uploaded only when
        they changed."""
        src = getattr(self, "_attach_src", None)
        if src is None or src.size == 0 or self._attach_tgt is None or self.bone_pos.shape[0] == 0:
            return
        last = getattr(self, "_attach_bone_last", None)
        if last is not None and last.shape == self.bone_pos.shape and np.array_equal(last, self.bone_pos):
            return
        self._attach_bone_last = self.bone_pos.copy()
        lib_idx = torch.from_numpy(self.layout.inv[src].astype(np.int64)).to(self.device)
        tgt = torch.from_numpy(np.ascontiguousarray(self.bone_pos[self._attach_tgt_idx], np.float32)).to(self.device)
        with torch.cuda.stream(self._stream):
            self._attach_tgt[lib_idx, :3] = tgt

    def build_constraints(self) -> None:
        """build_constraints (musclesim.py:365-389): the constraint blocks
        collected again (with the current point attributes in ``self.geo`` and
        bone points in ``self.bone_pos``) and the device rebuilt; the state
        carries over."""
        table = collect_raw_constraints(self.pos0_np, self.tet_np, self.constraint_configs,
                                        getattr(self, "_tet_masks", None))
        attach = self._bone_attach_rows(self.pos0_np, self.tet_np)
        if attach is not None:
            table = ConstraintTable.concat([table, attach])
        self.raw_constraints = table.sorted_by_type()
        self._attach_bone_last = None
        self.rebuild_constraints()

    def rebuild_constraints(self, extra_constraints=None) -> None:
        """musclesim.py:289-321: the constraint table rebuilt from the raw
        constraints plus ``extra_constraints`` (dicts in the reference's schema,
        e.g. ATTACH rows added after the build), sorted by type.  The device
        layout is rebuilt; positions, previous positions, velocities and the
        stopped flags carry over."""
        from .builder import constraints_from_dicts
        extra = list(extra_constraints or [])
        parts = [self.raw_constraints] + ([constraints_from_dicts(extra)] if extra else [])
        table = ConstraintTable.concat(parts).sorted_by_type()
        pos, prev, vel = self.positions_np(), self.pprev.numpy(), self.vel.numpy()
        self.release_graphs()
        self._setup_device(stopped=self._stopped_user.copy(), table=table, **self._setup_kw)
        self.set_positions(prev, also_prev=True)
        self.set_positions(pos)
        self.set_velocities(vel)

    # ---------------------------------------------------------------- program
    def build_program(self):
        """Default program (musclesim.py:107-130): integrate_phase, solve_phase,
        finalize_phase."""
        s = self

        def integrate_phase():
            s.integrate()
            s.apply_pintotarget()
            s.clear()

        def solve_phase():
            s.solve_constraints(run_extras=False)
            s.apply_dP()
            s.solve_extras()

        def finalize_phase():
            s.post_smooth()
            s.freeze_near_inverted()
            s.repair_inverted_tets()
            s.apply_pintotarget()
            s.update_velocities()

        self.program = [integrate_phase, solve_phase, finalize_phase]

    def _hooks(self) -> bool:
        return (bool(getattr(self, "constraint_solvers", None)) or int(self._option("post_smooth_iters", 0)) > 0
                or (float(self._option("repair_alpha", 0.0)) > 0.0 and int(self._option("repair_iters", 0)) > 0))

    def _frame_fused(self) -> None:
        """One frame, fused: [predict] (tile pass + boundary finish) ... with the
        velocity update of substep s folded into the prediction of s+1."""
        n = self.num_substeps
        for sub in range(n):
            ops = capi.OP_PREDICT | (capi.OP_VELOCITY if sub > 0 else 0)
            self._vstep(ops)
            if self.n_cons > 0:
                self._fused_iteration()
        self._vstep(capi.OP_VELOCITY)

    def step(self):
        """One frame (musclesim.py:136-142): the bone-attach targets follow the
        bones, then the substeps."""
        self._check_status()
        self.update_attach_targets()
        if self._hooks():
            if getattr(self, "program", None) is None:
                self.build_program()
            self.run_program()
        else:
            self._graph("frame", self._frame_fused)
        self._post_status()
        self.step_cnt += 1

    def step_eager(self):
        """One frame through the phase program (no graph, unfused primitives)."""
        self.update_attach_targets()
        if getattr(self, "program", None) is None:
            self.build_program()
        self.run_program()
        self.step_cnt += 1

    def set_fiber_activation(self, acti_np) -> None:
        """Per-tet activation in the user's tet order (mg.py:1098-1111)."""
        if self._t_act is None:
            raise RuntimeError("set_fiber_activation requires an aniso_arap constraint")
        import torch
        a = np.ascontiguousarray(np.asarray(acti_np, np.float32)[self.layout.tet_perm])
        with torch.cuda.stream(self._stream):
            self._t_act.copy_(torch.from_numpy(a).to(self.device), non_blocking=False)
        self._stream.synchronize()
