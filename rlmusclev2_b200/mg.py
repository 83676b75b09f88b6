"""MultiGridSim (the reference's OneWaySim successor, src/muscle/mg/mg.py:85-1443)
on the sm_100a engine.

Same JSON schema (``constraints[]`` blocks looked up by name with ``enable``
toggles, solver keys at the top level).  The rest mesh comes from a seeded
synthetic generator (``cfg["synthetic"]``) because the reference's humanV2
assets are not available.  Kinematic targets (mg.py:436-446):
target_mode="mesh" binds every vertex to the closest point of the bone
surfaces at the start frame and rides (optionally slides along) them
(mg.py:1117-1174; the synthetic bones are capsule surfaces posed rigidly);
target_mode="lbs" gives every vertex a smooth target blended between the two
bones at its muscle's ends, computed on the device from the bone poses (the
synthetic counterpart of the reference's precomputed LBS target sequence), or,
with ``lbs_target_npz``, read from such a sequence file (points (F, NV, 3),
frames); target_mode="points" reads the cons_<frame>.geo pin-to-target frames.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import torch

from . import _capi as capi
from .builder import ConstraintTable, collect_raw_constraints, create_attach_constraints, lumped_mass, tet_rest_data
from .collision import GridSdfCollider, UdcfDcdCollider, UdcfParams
from .meshgen import Scene, humanv2_scene
from .musclesim import MuscleSim


def find_constraint(cfg: dict, name: str) -> dict | None:
    """mg.py:71-82: the constraint block named ``name`` unless ``enable`` is false."""
    for c in cfg.get("constraints", []):
        if c.get("name") == name:
            return c if c.get("enable", True) else None
    return None


def load_config(config_path: str) -> dict:
    """mg.py:1437-1443: JSON scene config with cwd-resolved relative paths."""
    cfg = json.load(open(config_path))
    for key in ("geo_dir", "cons_dir", "rest_path", "fascia_path"):
        if key in cfg and not Path(cfg[key]).is_absolute():
            cfg[key] = str(Path.cwd() / cfg[key])
    return cfg


def scene_from_cfg(cfg: dict) -> Scene:
    syn = dict(cfg.get("synthetic") or {})
    kind = syn.pop("kind", "humanv2")
    if kind == "humanv2":
        return humanv2_scene(**syn)
    if kind == "batched_boxes":
        from .meshgen import batched_box_scene
        return batched_box_scene(**syn)
    raise ValueError(f"unknown synthetic scene kind {kind!r}")


class MultiGridSim(MuscleSim):
    """One-way pin-to-target XPBD solver (mg.py:85)."""

    #: iterations followed by a hook (the DCD) as one-iteration persistent launches
    #: (one kernel instead of two; 1 % slower on config 3's 535k-tet scene, whose
    #: one-iteration launches pay the cooperative launch and a grid barrier)
    persistent_between_hooks = False

    def __init__(self, cfg: dict, device: str | None = "cuda:0", scene: Scene | None = None):
        self.cfg = cfg
        self._device_str = device or "cuda:0"
        self.quasi_static = bool(cfg.get("quasi_static", False))
        self._gravity_vec = tuple(float(x) for x in cfg.get("gravity", [0.0, 0.0, 0.0]))
        _arap = find_constraint(cfg, "arap")
        if _arap is None:
            raise ValueError("constraints[] must define an 'arap' entry (the muscle ARAP-SVD shape match)")
        self.mu = float(_arap["stiffness"])
        self._arap_damp = float(_arap.get("dampingratio", 0.0))
        _snh = find_constraint(cfg, "snh")
        self.use_snh = _snh is not None
        self.snh_mu = float(_snh.get("mu", _snh.get("stiffness", self.mu))) if _snh else 0.0
        self.snh_lam = float(_snh.get("lam", 1.0e8)) if _snh else 0.0
        self.snh_damp = float(_snh.get("dampingratio", self._arap_damp)) if _snh else 0.0
        self.snh_region = str(_snh.get("region", "all")) if _snh else "all"
        self.omega = float(cfg["omega"])
        self.dt_frame = float(cfg["delta_t"])
        self.nsubsteps = int(cfg["nsubsteps"])
        self.num_substeps = self.nsubsteps
        # soft pin of every constraint point toward its bone target after the hard
        # pin, once per kinematic step (mg.py:133, 1386-1397); 0 = off
        self.presubframe_pintotarget = float(cfg.get("presubframe_pintotarget", 0.0))
        self.fine_iters = int(cfg["fine_iterations"])
        # density: total_mass spread over the signed rest volume (mg.py:736-740),
        # or a fixed "density" (kg/m^3, the MuscleSim.from_procedural form)
        self.total_mass = float(cfg.get("total_mass", 0.0))
        self._fixed_density = cfg.get("density")
        self.dt = self.dt_frame / self.nsubsteps
        self.end_frame = int(cfg.get("end_frame", 90))
        self.start_frame = int(cfg.get("start_frame", 1))
        self.use_multigrid = bool(cfg.get("use_multigrid", False))
        self.mg_mode = str(cfg.get("mg_mode", "hpbd")).lower()
        if self.mg_mode not in ("projection", "hpbd"):
            raise ValueError(f"mg_mode must be 'projection' or 'hpbd', got {self.mg_mode!r}")
        self.mg_coarse_iters = int(cfg.get("mg_coarse_iters", 15))
        _vol = find_constraint(cfg, "volume")
        self.use_volume = _vol is not None
        self.volume_stiffness = float(_vol["stiffness"]) if _vol else 1.0e10
        self.volume_damp = float(_vol.get("dampingratio", 0.0)) if _vol else 0.0
        _fib = find_constraint(cfg, "fiber")
        self.use_fiber = _fib is not None
        self.fiber_model = str((_fib or {}).get("fiber_model", "aniso_arap"))
        self.fiber_stiffness = float((_fib or {}).get("stiffness", 1.0e8))
        self.fiber_damp = float((_fib or {}).get("dampingratio", 0.0))
        self.contraction_ratio = float((_fib or {}).get("contraction_ratio", 0.4))
        self.fiber_region = str((_fib or {}).get("region", "all"))
        if self.use_fiber and self.fiber_model != "aniso_arap":
            raise NotImplementedError(f"fiber_model={self.fiber_model!r} is not on the sm_100a path "
                                      "(supported: 'aniso_arap')")
        # asset_scale (util/bone_source.py:60-66, 301-315; mg.py:299-305): a
        # uniform scale of the USD rest mesh and of the bone_<frame>.geo
        # surfaces on load (0.01 for a centimetre asset); a .geo rest is not scaled
        self.asset_scale = float(cfg.get("asset_scale", 1.0))
        if scene is None and "synthetic" not in cfg and cfg.get("rest_path"):
            rp = Path(cfg["rest_path"])
            if rp.suffix.lower() not in (".geo", ".usda", ".usd"):
                raise NotImplementedError(f"rest mesh {rp.name}: Houdini .geo assets and text USD layers are read")
            if not rp.exists():
                raise FileNotFoundError(f"rest_path {rp} does not exist")
            if rp.suffix.lower() == ".geo":
                from .geo import scene_from_geo
                scene = scene_from_geo(rp)
            else:
                from .usd import scene_from_usda
                if cfg.get("muscle_prim_root"):
                    raise NotImplementedError("muscle_prim_root (merging every TetMesh under a root) is not read; "
                                              "name one TetMesh with muscle_prim_path")
                # the layer's points as authored (no xform ops are applied; usd_local_space)
                scene = scene_from_usda(rp, cfg.get("muscle_prim_path") or cfg.get("rest_prim_path"))
                scene.verts = self._asset_scaled(scene.verts)
        self.scene = scene if scene is not None else scene_from_cfg(cfg)
        sc = self.scene
        # kinematic targets (mg.py:436-446)
        self.target_mode = str(cfg.get("target_mode", "lbs"))
        self.use_sliding = bool(cfg.get("use_sliding", False))
        self.slide_range = float(cfg.get("slide_range", 0.005))
        self.slide_interval = int(cfg.get("slide_interval", 1))
        if self.target_mode not in ("mesh", "lbs", "points"):
            raise NotImplementedError(f"target_mode={self.target_mode!r} is not on the sm_100a path "
                                      "(supported: 'mesh', 'lbs', 'points')")
        self.cons_dir = cfg.get("cons_dir")
        if self.target_mode == "points" and not self.cons_dir:
            raise ValueError("target_mode='points' reads cons_<frame>.geo frames: set cons_dir")
        if self.use_sliding and self.target_mode != "mesh":
            raise ValueError("use_sliding=true requires target_mode='mesh' (mg.py:438-440)")
        self.pos0_np = sc.verts.astype(np.float32)
        self.tet_np = sc.tets.astype(np.int32)
        self.NV = self.n_verts = int(self.pos0_np.shape[0])
        self.NT = int(self.tet_np.shape[0])
        # target_mode="lbs" with lbs_target_npz: a precomputed target sequence
        # (F, NV, 3) for every vertex, read on the host (_build_lbs_target,
        # mg.py:1176-1198); without it the lbs targets are computed on the device
        self.lbs_target_npz = cfg.get("lbs_target_npz") if self.target_mode == "lbs" else None
        if self.lbs_target_npz:
            with np.load(self.lbs_target_npz) as z:
                self._lbs_pts = np.asarray(z["points"], np.float32)
                self._lbs_f0 = int(np.asarray(z["frames"], np.int32)[0])
            if self._lbs_pts.ndim != 3 or self._lbs_pts.shape[1:] != (self.NV, 3):
                raise ValueError(f"lbs_target_npz points {self._lbs_pts.shape} != (F, NV={self.NV}, 3)")
        # targets that come from the host every frame (cons frames or the lbs file)
        self._host_tgt = self.target_mode == "points" or bool(self.lbs_target_npz)
        # the solve is the Jacobi projection (mg.py:353-354 read use_jacobi,
        # default true, and use_colored_gs, default false): the Gauss-Seidel
        # variants are refused rather than silently replaced
        if not bool(cfg.get("use_jacobi", True)) or bool(cfg.get("use_colored_gs", False)):
            raise NotImplementedError("use_jacobi=false / use_colored_gs=true select the reference's Gauss-Seidel "
                                      "solves, which are not on the sm_100a path (it runs the Jacobi projection)")
        self.use_jacobi = True
        self.use_colored_gs = False
        self.has_compressstiffness = False
        self.fiber_stiffness_scale = 1.0
        self.step_cnt = 0
        # constraint set (mg.py:374-399): SNH or ARAP-SVD, optional volume and fiber
        fascia = sc.tet_part < 0
        masks = {}
        if self.use_snh:
            cons = [dict(type="snh", name="snh", mu=self.snh_mu, lam=self.snh_lam, dampingratio=self.snh_damp)]
            if self.snh_region == "fascia":
                masks["snh"] = fascia
                masks["arap"] = ~fascia
                cons.append(dict(type="tetarapsvd", name="arap", stiffness=self.mu, dampingratio=self._arap_damp))
            elif self.snh_region != "all":
                raise ValueError(f"snh region must be 'all' or 'fascia', got {self.snh_region!r}")
        else:
            cons = [dict(type="tetarapsvd", name="arap", stiffness=self.mu, dampingratio=self._arap_damp)]
        if self.use_volume and not (self.use_snh and self.snh_region == "all"):
            cons.append(dict(type="volume", name="volume", stiffness=self.volume_stiffness,
                             dampingratio=self.volume_damp))
            if self.use_snh:
                masks["volume"] = ~fascia
        if self.use_fiber:
            cons.append(dict(type="aniso_arap", name="fiber", stiffness=self.fiber_stiffness,
                             dampingratio=self.fiber_damp))
            if self.fiber_region == "aniso_muscle":
                masks["fiber"] = sc.tet_part == sc.aniso_muscle
            elif self.fiber_region != "all":
                raise ValueError(f"fiber region must be 'all' or 'aniso_muscle', got {self.fiber_region!r}")
        self.constraint_configs = cons
        table = collect_raw_constraints(self.pos0_np, self.tet_np, cons, tet_masks=masks)
        # density = total_mass / sum(signed V0) (mg.py:736-740), mass = |V| rho / 4
        _, V0, valid = tet_rest_data(self.pos0_np, self.tet_np)
        if self._fixed_density is not None:
            self.density = float(self._fixed_density)
        else:
            self.density = self.total_mass / float(max(V0[valid].astype(np.float64).sum(), 1e-30))
        mass, rest_volume = lumped_mass(self.pos0_np, self.tet_np, self.density)
        self.total_rest_volume = float(rest_volume.astype(np.float64).sum())
        # pins (muscleToBonePin, mg.py:486-535) and belly attach (mg.py:700-723)
        self.NCONS = self.NV
        self._pin_pts_np = np.arange(self.NV, dtype=np.int64)
        _pin = find_constraint(cfg, "muscleToBonePin")
        active = np.zeros(self.NV, np.int32)
        if _pin is not None:
            region = str(_pin.get("region", "tendonmask")).lower()
            if region == "full":
                active[:] = 1
            elif region == "tendonmask":
                thr = _pin.get("tendon_pin_threshold")
                if thr is None:
                    raise ValueError("muscleToBonePin region='tendonmask' requires tendon_pin_threshold")
                active = (sc.v_tendon > float(thr)).astype(np.int32)
            elif region == "pinmask":
                active[:] = 0  # the synthetic rest carries no authored pinmask
            else:
                raise ValueError(f"muscleToBonePin 'region' must be 'full', 'tendonmask' or 'pinmask', got {region!r}")
        if self.target_mode == "points":
            # pin-to-target topology from the start frame's cons file (mg.py:448-458):
            # only its points are pinned or attached, offset by rest - target_pos
            from .geo import GeoFile
            cons0 = GeoFile(Path(self.cons_dir) / f"cons_{self.start_frame}.geo")
            self._cons_pts = cons0.pts.astype(np.int64)
            self._cons_cache = {}
            in_cons = np.zeros(self.NV, bool)
            in_cons[self._cons_pts] = True
            active = (active.astype(bool) & in_cons).astype(np.int32)
        elif self.lbs_target_npz:
            self._cons_pts = np.arange(self.NV, dtype=np.int64)  # every vertex, rest_offset 0
        self.pin_active_np = active
        _belly = find_constraint(cfg, "belly_attach")
        self._belly_enabled = _belly is not None
        self.pin_attach_stiffness = float(_belly["stiffness"]) if _belly else 0.0
        self.pin_attach_damp = float(_belly.get("dampingratio", 0.0)) if _belly else 0.0
        self.rest_offset_np = np.zeros((self.NV, 3), np.float32)
        if self.target_mode == "points":
            self.rest_offset_np[self._cons_pts] = (self.pos0_np[self._cons_pts] - cons0.target_pos).astype(np.float32)
        target0 = self._host_targets(self.start_frame)
        parts = [table]
        if self._belly_enabled:
            belly = np.nonzero(active == 0)[0]
            if self.target_mode == "points":
                belly = belly[in_cons[belly]]
            parts.append(create_attach_constraints(belly, target0[belly] + self.rest_offset_np[belly], 0.0,
                                                   self.pin_attach_stiffness, self.pin_attach_damp))
        table = ConstraintTable.concat(parts).sorted_by_type()
        self.raw_constraints = table
        self._pin_user = (active != 0, target0 + self.rest_offset_np, active)
        self._has_pins = bool(active.any())
        tendon_tet = (sc.v_tendon[self.tet_np].astype(np.float32).sum(1) / np.float32(4.0)).astype(np.float32)
        self._setup_device(self._device_str, mass=mass, stopped=np.zeros(self.NV, np.int32), table=table,
                           v_fiber=sc.v_fiber, tet_tendonmask=tendon_tet, dt=self.dt,
                           gravity_vec=self._gravity_vec, veldamping=float(cfg.get("veldamping", 0.0)),
                           quasi_static=self.quasi_static, omega=1.0, contraction_ratio=self.contraction_ratio,
                           fiber_stiffness_scale=self.fiber_stiffness_scale, tile_tets=cfg.get("tile_tets"),
                           vert_group=getattr(sc, "vert_inst", None))
        self._setup_kinematics()
        self._setup_m2m_glue()
        self._setup_fascia()
        self.collision_solvers_iter = []
        self.mg = None
        if self.use_multigrid:
            from .multigrid import DeviceMultigrid
            self.mg = DeviceMultigrid(self, spacing=float(cfg.get("mg_cage_spacing", 0.016)))
        self.collision_solvers = []
        coll = (cfg.get("demo") or {}).get("collision") or {}
        if coll.get("enabled", False) and sc.n_bones == 0:
            raise ValueError("demo.collision needs capsule bones; this scene has none (disable it)")
        if coll.get("enabled", False):
            self.bone_collider = GridSdfCollider(
                self, sc.bone_center, sc.bone_axis, sc.bone_half, sc.bone_radius, res=int(coll.get("sdf_res", 256)),
                contact_offset=float(coll.get("contact_offset", 0.0)), max_push=float(coll.get("max_push", -1.0)))
            self.bone_collider.transforms = self._bone_tr
            self.collision_solvers.append(self.bone_collider)
        sc_cfg = (cfg.get("demo") or {}).get("self_collision") or {}
        if str(sc_cfg.get("method", "none")).lower() == "udcf":
            prm = UdcfParams(multiplier=float(sc_cfg.get("multiplier", 1.01)),
                             friction_static=float(sc_cfg.get("friction_static", 0.5)),
                             friction_dynamic=float(sc_cfg.get("friction_dynamic", 0.4)),
                             offset=float(sc_cfg.get("offset", 1e-6)), thickness=float(sc_cfg.get("thickness", 0.0)),
                             max_pairs=int(sc_cfg.get("max_pairs", 1 << 22)),
                             max_contacts=int(sc_cfg.get("max_contacts", 1 << 20)),
                             allow_self=bool(sc_cfg.get("allow_self", True)), max_push=float(sc_cfg.get("max_push", 0.0)),
                             bvh_rebuild_every=int(sc_cfg.get("bvh_rebuild_every", 1)))
            self.dcd = UdcfDcdCollider(self, sc.surface_tris, prm)
            self.collision_solvers_iter.append(self.dcd.solve)
        self._frame_loaded = None

    # ----------------------------------------------------------- kinematics
    def _cons_targets(self, frame: int) -> np.ndarray:
        """Targets of ``frame`` in user order: the cons file's target_pos on its
        points, the rest position elsewhere (load_frame_targets, mg.py:1238-1250;
        frames are read once and kept).  The pins and attachments add the rest
        offset."""
        if frame not in self._cons_cache:
            from .geo import read_cons_frame
            self._cons_cache[frame] = read_cons_frame(self.cons_dir, int(frame)).astype(np.float32)
        tgt = self.pos0_np.copy()
        tgt[self._cons_pts] = self._cons_cache[frame]
        return tgt

    def _lbs_targets(self, frame: float) -> np.ndarray:
        """_update_lbs_target (mg.py:1200-1214): the sequence's frame, clamped
        to its range, linearly blended between the two frames around a
        fractional frame (the weight is a float64 scalar, so the blend runs in
        FP64 and is rounded to FP32 once)."""
        f = float(frame)
        n = self._lbs_pts.shape[0]
        lo = min(max(int(np.floor(f)) - self._lbs_f0, 0), n - 1)
        hi = min(max(int(np.ceil(f)) - self._lbs_f0, 0), n - 1)
        if lo == hi:
            return self._lbs_pts[lo].copy()
        w = f - np.floor(f)
        return ((1.0 - w) * self._lbs_pts[lo] + w * self._lbs_pts[hi]).astype(np.float32)

    def _host_targets(self, frame: float) -> np.ndarray:
        if self.lbs_target_npz:
            return self._lbs_targets(frame)
        if self.target_mode == "points":
            return self._cons_targets(int(frame))
        if self.target_mode == "mesh":
            if frame != self.start_frame:
                raise ValueError("host targets of the surface binding exist for the start frame only")
            return self.pos0_np.copy()  # the bind reconstructs the rest pose on the start-frame bones
        return self.scene.targets(frame)

    def _setup_kinematics(self) -> None:
        L = self.layout
        dev = self.device
        nb = self.scene.n_bones
        self._bone_tr = torch.zeros((nb, 12), dtype=torch.float32, device=dev)
        self._bone_tr_host = torch.zeros((nb, 12), dtype=torch.float32).pin_memory()
        self._vert_bone = torch.from_numpy(np.ascontiguousarray(self.scene.vert_bone[L.perm], np.int32)).to(dev)
        self._vert_bw = torch.from_numpy(np.ascontiguousarray(self.scene.vert_bw[L.perm], np.float32)).to(dev)
        r4 = np.zeros((self.NV, 4), np.float32)
        r4[:, :3] = self.pos0_np
        self._rest4 = torch.from_numpy(r4[L.perm]).to(dev)
        self._tet_perm_d = torch.from_numpy(L.tet_perm.astype(np.int32)).to(dev)
        self._vinv_d = torch.from_numpy(L.inv.astype(np.int32)).to(dev)
        self._act_user = torch.zeros(self.NT, dtype=torch.float32, device=dev)
        self._act_host = torch.zeros(self.NT, dtype=torch.float32).pin_memory()
        self._pos_user = torch.zeros((self.NV, 3), dtype=torch.float32, device=dev)
        self._pos_host = torch.zeros((self.NV, 3), dtype=torch.float32).pin_memory()
        # One event per pinned staging buffer: a buffer is refilled only after
        # its own previous copy has been consumed, so the activation upload and
        # the target upload of one frame do not wait on each other.
        self._act_event = torch.cuda.Event()
        self._act_event.record(self._stream)
        self._h2d_event = torch.cuda.Event()
        self._h2d_event.record(self._stream)
        self._presub_idx = None  # constraint points of the soft pin: all vertices
        if self._host_tgt:
            self._pts_tgt = torch.zeros((self.NV, 3), dtype=torch.float32, device=dev)
            self._pts_host = torch.zeros((self.NV, 3), dtype=torch.float32).pin_memory()
        if self.target_mode == "points":
            self._presub_idx = torch.from_numpy(L.inv[self._cons_pts].astype(np.int32)).to(dev)
        if self.target_mode == "mesh":
            self._setup_surface_binding()

    def _setup_surface_binding(self) -> None:
        """_build_bone_slide_binding (mg.py:1117-1158): the bone surfaces posed
        at the start frame, every vertex's rest position bound to its closest
        surface point (face, barycentric, offset in the face frame); the current
        binding starts at that anchor."""
        dev = self.device
        self._bone_dir = self.cfg.get("bone_dir")
        if self._bone_dir and not Path(self._bone_dir).is_dir():
            self._bone_dir = None
        if self._bone_dir:
            # GeoBoneSource (util/bone_source.py:84-116): triangles of bone_<start>.geo,
            # positions of bone_<frame>.geo uploaded every frame
            from .geo import GeoFile
            g0 = GeoFile(Path(self._bone_dir) / f"bone_{self.start_frame}.geo")
            bv = self._asset_scaled(g0.positions)
            bt = np.asarray(g0.tet_indices, np.int32).reshape(-1, 3)
            bvb = np.zeros(bv.shape[0], np.int32)
            self._bone_frames = {}
            self._bs_host = torch.zeros((bv.shape[0], 4), dtype=torch.float32).pin_memory()
        elif hasattr(self.scene, "bone_surface") and self.scene.n_bones > 0:
            bv, bt, bvb = self.scene.bone_surface()
        else:
            raise NotImplementedError("target_mode='mesh' needs bone surfaces: a bone_dir of bone_<frame>.geo "
                                      "files or a scene with capsule bones")
        r4 = np.zeros((bv.shape[0], 4), np.float32)
        r4[:, :3] = bv
        self._bs_rest4 = torch.from_numpy(r4).to(dev)
        self._bs_pos4 = torch.zeros_like(self._bs_rest4)
        self._bs_tris = torch.from_numpy(np.ascontiguousarray(bt, np.int32)).to(dev)
        self._bs_vbone = torch.from_numpy(np.ascontiguousarray(bvb, np.int32)).to(dev)
        self._slide_max_dist = float(self.slide_range + 1.0)  # mg.py:1131
        nv = self.NV
        self._anchor_face = torch.zeros(nv, dtype=torch.int32, device=dev)
        self._anchor_uv = torch.zeros((nv, 2), dtype=torch.float32, device=dev)
        self._local4 = torch.zeros((nv, 4), dtype=torch.float32, device=dev)
        self.load_frame_targets(self.start_frame)
        self._pose_bone_surface()
        capi.check(self._lib.xpbd_bone_bind(nv, C.c_void_p(self._rest4.data_ptr()), int(bv.shape[0]),
                                            C.c_void_p(self._bs_pos4.data_ptr()), int(bt.shape[0]),
                                            C.c_void_p(self._bs_tris.data_ptr()), C.c_float(self._slide_max_dist),
                                            C.c_void_p(self._anchor_face.data_ptr()),
                                            C.c_void_p(self._anchor_uv.data_ptr()),
                                            C.c_void_p(self._local4.data_ptr()), self._sp))
        with torch.cuda.stream(self._stream):
            self._bind_face = self._anchor_face.clone()
            self._bind_uv = self._anchor_uv.clone()
        self._reproject = False

    def _setup_m2m_glue(self) -> None:
        """_build_m2m_glue (mg.py:581-660) when the config has a
        muscleToMuscleGlue block.  The per-vertex muscle id comes from the
        scene (``vert_muscle``, else the part of the vertex's tets); the enable
        mask from the scene's ``m2m_mask`` or, for the synthetic scenes, the
        block's ``region``: "all" muscle vertices, their "surface" ones, or the
        "interface" ones (a vertex of another muscle within ``distance``), the
        stand-in for the authored muscletomuscleglue mask."""
        from .glue import build_m2m_pairs
        self.n_m2m = 0
        g = find_constraint(self.cfg, "muscleToMuscleGlue")
        if g is None:
            return
        sc = self.scene
        vm = getattr(sc, "vert_muscle", None)
        if vm is None:
            vm = np.full(self.NV, -1, np.int64)
            part = np.asarray(sc.tet_part)
            keep = part >= 0
            vm[self.tet_np[keep].reshape(-1)] = np.repeat(part[keep], 4)
        dist = float(g.get("distance", -1.0))
        radius = dist if dist > 0.0 else 0.01
        mask = getattr(sc, "m2m_mask", None)
        if mask is None:
            region = str(g.get("region", "all"))
            mask = (vm >= 0).astype(np.float32)
            if region == "surface":
                on = np.zeros(self.NV, np.float32)
                on[np.unique(sc.surface_tris)] = 1.0
                mask = mask * on
            elif region == "interface":
                from scipy.spatial import cKDTree
                on = np.zeros(self.NV, np.float32)
                for m in np.unique(vm[vm >= 0]):
                    mine, other = np.nonzero(vm == m)[0], np.nonzero((vm >= 0) & (vm != m))[0]
                    if other.size:
                        d, _ = cKDTree(self.pos0_np[other]).query(self.pos0_np[mine])
                        on[mine[d <= radius]] = 1.0
                mask = on
            elif region != "all":
                raise ValueError(f"muscleToMuscleGlue 'region' must be 'all', 'surface' or 'interface', "
                                 f"got {region!r}")
        a, b, rest = build_m2m_pairs(self.pos0_np, vm, mask, float(g.get("mask_threshold", 0.5)), radius,
                                     int(g.get("knn", 8)))
        if a.size == 0:
            return
        stiff = max(float(g.get("stiffness", 1.0e4)) * float(g.get("stiffness_scale", 1.0)), 1.0e-30)
        inv = self.layout.inv
        dev = self.device
        self.m2m_pairs_user = (a, b)
        self._m2m_a = torch.from_numpy(inv[a].astype(np.int32)).to(dev)
        self._m2m_b = torch.from_numpy(inv[b].astype(np.int32)).to(dev)
        self._m2m_rest = torch.from_numpy(rest).to(dev)
        self._m2m_comp = torch.full((a.size,), 1.0 / stiff, dtype=torch.float32, device=dev)
        self.n_m2m = int(a.size)

    def _setup_fascia(self) -> None:
        """The fascia shell sub-solver (mg.py:556-566) in "ride" or "squeeze"
        mode: the shell from ``fascia_path`` (a .geo read by geo.GeoFile) or,
        for the synthetic scenes, a shell offset from the muscle surface
        (meshgen.fascia_shell)."""
        self.fascia = None
        if not bool(self.cfg.get("use_fascia", False)):
            return
        mode = str(self.cfg.get("fascia_mode", "squeeze"))
        if mode not in ("ride", "squeeze"):
            raise NotImplementedError(f"fascia_mode={mode!r} is not on the sm_100a path (supported: 'ride', "
                                      "'squeeze')")
        if (np.asarray(self.scene.tet_part) < 0).any():
            raise ValueError("use_fascia needs a scene without merged fascia tets (fascia_tets=0)")
        from .fascia import FasciaRide
        from .meshgen import fascia_shell
        path = self.cfg.get("fascia_path")
        g = None
        if path and Path(path).exists():
            from .geo import GeoFile
            from .meshgen import orient_tets
            g = GeoFile(path)
            fv = g.positions
            ft = orient_tets(fv, np.asarray(g.tet_indices, np.int64)).astype(np.int32)
        else:
            fv, ft = fascia_shell(self.pos0_np, self.scene.surface_tris,
                                  float(self.cfg.get("fascia_gap", 0.001)), float(self.cfg.get("fascia_thickness", 0.003)))
        snh = find_constraint(self.cfg, "fascia_snh") or {}
        glue = find_constraint(self.cfg, "fascia_glue") or {}
        if mode == "squeeze":
            from .fascia import FasciaSqueeze
            arap = find_constraint(self.cfg, "fascia_arap") or {}
            vol = find_constraint(self.cfg, "fascia_volume") or {}
            anchor = find_constraint(self.cfg, "fascia_anchor") or {}
            ak = float(arap.get("stiffness", -1.0))
            if ak < 0.0:  # the asset's solidshapestiffness (fascia.py:244-248)
                if g is None or not g.has_point_attr("solidshapestiffness"):
                    raise ValueError("fascia_arap.stiffness is required without a 'solidshapestiffness' attribute")
                ak = float(g.point_attr("solidshapestiffness").mean())
            gk = glue.get("stiffness")
            if gk is None:  # the asset's tissuetomusclestiffness (fascia.py:433-438)
                if g is None or not g.has_point_attr("tissuetomusclestiffness"):
                    raise ValueError("fascia_glue.stiffness is required without a 'tissuetomusclestiffness' attribute")
                gk = float(g.point_attr("tissuetomusclestiffness").mean())
            rigid = g.point_group("rigid") if (g is not None and g.has_point_group("rigid")) else None
            self.fascia = FasciaSqueeze(
                self, fv, ft, rest_scale=float(arap.get("rest_scale", 0.95)), arap_k=ak,
                arap_damp=float(arap.get("dampingratio", 0.0)), vol_k=float(vol.get("stiffness", 1.0e10)),
                vol_damp=float(vol.get("dampingratio", 0.0)),
                glue_k=float(gk) * float(glue.get("stiffness_scale", 0.001)),
                total_mass=float(self.cfg.get("fascia_total_mass", self.total_mass)),
                iterations=int(glue.get("iterations", self.fine_iters)), anchor_count=int(anchor.get("count", 256)),
                rigid=rigid)
            return
        self.fascia = FasciaRide(self, fv, ft, snh_mu=float(snh.get("mu", 1.0e3)), snh_lam=float(snh.get("lam", 1.0e8)),
                                 snh_damp=float(snh.get("dampingratio", 0.0)),
                                 total_mass=float(self.cfg.get("fascia_total_mass", self.total_mass)),
                                 iterations=int(glue.get("iterations", self.fine_iters)),
                                 bind_max_dist=float(self.cfg.get("fascia_bind_max_dist", 0.05)))

    def _solve_m2m_glue(self) -> None:
        """_solve_m2m_glue (mg.py:662-670): one glue step with the config's omega."""
        if not self.n_m2m:
            return
        capi.check(self._lib.xpbd_m2m_glue(self.n_m2m, C.c_void_p(self._m2m_a.data_ptr()),
                                           C.c_void_p(self._m2m_b.data_ptr()), C.c_void_p(self._m2m_rest.data_ptr()),
                                           C.c_void_p(self._m2m_comp.data_ptr()), C.c_void_p(self._pos4.data_ptr()),
                                           C.c_float(self.dt), C.c_float(self.omega), self._sp))

    def _m2m_iteration(self) -> None:
        """One fine iteration in the reference's order with the glue between the
        averaged correction and the re-pin (mg.py:1346-1355)."""
        self.clear()
        self.solve_constraints(run_extras=False)
        self.apply_dP()
        self._solve_m2m_glue()
        self.apply_pintotarget()

    def _asset_scaled(self, arr) -> np.ndarray:
        """Positions times asset_scale in FP32 (unchanged at 1)."""
        arr = np.asarray(arr, np.float32)
        if self.asset_scale == 1.0:
            return arr
        return np.ascontiguousarray((arr * np.float32(self.asset_scale)).astype(np.float32))

    def _upload_bone_frame(self, frame: int) -> None:
        """bone_<frame>.geo positions into the bone-surface buffer (one pinned H2D copy)."""
        from .geo import read_geo_attr
        if frame not in self._bone_frames:
            self._bone_frames[frame] = self._asset_scaled(
                read_geo_attr(Path(self._bone_dir) / f"bone_{int(frame)}.geo", "P"))
        self._h2d_event.synchronize()
        self._bs_host.numpy()[:, :3] = self._bone_frames[frame]
        with torch.cuda.stream(self._stream):
            self._bs_pos4.copy_(self._bs_host, non_blocking=True)
        self._h2d_event.record(self._stream)

    def _pose_bone_surface(self) -> None:
        if self._bone_dir:
            return  # the frame's bone positions were uploaded by load_frame_targets
        capi.check(self._lib.xpbd_bone_surface_pose(int(self._bs_rest4.shape[0]), C.c_void_p(self._bs_rest4.data_ptr()),
                                                    C.c_void_p(self._bs_vbone.data_ptr()), self.scene.n_bones,
                                                    C.c_void_p(self._bone_tr.data_ptr()),
                                                    C.c_void_p(self._bs_pos4.data_ptr()), self._sp))

    def load_frame_targets(self, frame: float) -> None:
        """Bone poses of ``frame`` -> device (one pinned H2D copy), then the
        per-vertex pin/attach targets on the device (mg.py:1386-1407); with
        target_mode="points" the frame's cons targets, with lbs_target_npz the
        file's targets, instead."""
        if self._host_tgt:
            tgt = (self._host_targets(frame) + self.rest_offset_np)[self.layout.perm]
            self._h2d_event.synchronize()
            self._pts_host.copy_(torch.from_numpy(np.ascontiguousarray(tgt, np.float32)))
            with torch.cuda.stream(self._stream):
                self._pts_tgt.copy_(self._pts_host, non_blocking=True)
            self._h2d_event.record(self._stream)
            self._frame_loaded = frame
            self._reproject = False
            return
        if self.target_mode == "mesh" and getattr(self, "_bone_dir", None):
            self._upload_bone_frame(int(frame))
        else:
            T = self.scene.bone_transforms(frame).reshape(self.scene.n_bones, 12).astype(np.float32)
            self._h2d_event.synchronize()  # the previous copy has consumed the pinned buffer
            self._bone_tr_host.numpy()[:] = T
            with torch.cuda.stream(self._stream):
                self._bone_tr.copy_(self._bone_tr_host, non_blocking=True)
            self._h2d_event.record(self._stream)
        self._frame_loaded = frame
        # _update_slide_target (mg.py:1160-1174): re-project every slide_interval frames
        self._reproject = bool(self.use_sliding and
                               (int(frame) - int(self.start_frame)) % max(1, self.slide_interval) == 0)

    def _targets_kernel(self) -> None:
        v = self._verts
        if self._host_tgt:
            with torch.cuda.stream(self._stream):
                for t in (self._pin_tgt, self._attach_tgt):
                    if t is not None:
                        t[:, :3].copy_(self._pts_tgt)
            return
        if self.target_mode == "mesh":
            self._pose_bone_surface()
            capi.check(self._lib.xpbd_bone_slide_targets(
                self.NV, C.c_void_p(self._pos4.data_ptr()), C.c_void_p(self._anchor_face.data_ptr()),
                C.c_void_p(self._anchor_uv.data_ptr()), C.c_void_p(self._bind_face.data_ptr()),
                C.c_void_p(self._bind_uv.data_ptr()), C.c_void_p(self._local4.data_ptr()),
                C.c_float(self.slide_range), int(self._reproject), C.c_float(self._slide_max_dist),
                int(self._bs_rest4.shape[0]), C.c_void_p(self._bs_pos4.data_ptr()), int(self._bs_tris.shape[0]),
                C.c_void_p(self._bs_tris.data_ptr()), v.pin_target, v.attach_target, self._sp))
            return
        capi.check(self._lib.xpbd_bone_targets(self.NV, self.scene.n_bones, C.c_void_p(self._bone_tr.data_ptr()),
                                               C.c_void_p(self._vert_bone.data_ptr()),
                                               C.c_void_p(self._vert_bw.data_ptr()),
                                               C.c_void_p(self._rest4.data_ptr()), v.pin_target, v.attach_target,
                                               self._sp))

    def set_fiber_activation(self, acti_np) -> None:
        """Per-tet activation in user tet order (mg.py:1098-1111): pinned H2D copy,
        then a device gather into the library's tet order."""
        if not self.use_fiber or self._t_act is None:
            raise RuntimeError("set_fiber_activation requires use_fiber=True.")
        a = np.asarray(acti_np, np.float32).reshape(-1)
        if a.shape[0] != self.NT:
            raise ValueError(f"activation has {a.shape[0]} entries, expected NT={self.NT}")
        self._act_event.synchronize()
        self._act_host.copy_(torch.from_numpy(a))  # multi-threaded host copy
        with torch.cuda.stream(self._stream):
            self._act_user.copy_(self._act_host, non_blocking=True)
        self._act_event.record(self._stream)
        capi.check(self._lib.xpbd_gather(self.NT, 1, C.c_void_p(self._tet_perm_d.data_ptr()),
                                         C.c_void_p(self._act_user.data_ptr()), 1, C.c_void_p(self._t_act.data_ptr()),
                                         1, self._sp))

    def positions_np(self) -> np.ndarray:
        """Positions in the user's vertex order: device gather, one D2H copy."""
        capi.check(self._lib.xpbd_gather(self.NV, 3, C.c_void_p(self._vinv_d.data_ptr()),
                                         C.c_void_p(self._pos4.data_ptr()), 4, C.c_void_p(self._pos_user.data_ptr()),
                                         3, self._sp))
        with torch.cuda.stream(self._stream):
            self._pos_host.copy_(self._pos_user, non_blocking=True)
        self.synchronize()  # raises on a fatal status bit of the frames before
        out = torch.empty((self.NV, 3), dtype=torch.float32)
        out.copy_(self._pos_host)  # multi-threaded host copy out of the pinned buffer
        return out.numpy()

    # -------------------------------------------------------------- program
    def apply_pintotarget(self) -> None:
        """Hard pin of the active tendon verts (mg.py:1251-1261)."""
        if self._has_pins:
            self._apply_all(capi.APPLY_PIN)

    # ----------------------------------------------------------- helpers
    def count_coarse_inverted(self) -> int:
        """count_coarse_inverted (mg.py:954-965): cage tets with det F <= 0 at the
        current cage positions; 0 without the hpbd cage."""
        if self.mg is None or self.mg.mode != "hpbd":
            return 0
        return int(self.mg.coarse.count_inverted())

    def belly_track_mm(self) -> tuple[float, float]:
        """belly_track_mm (mg.py:967-977): median and mean distance in mm from
        each constraint point to its bone-driven goal (target_pos + rest_offset);
        one device sync."""
        if self._pin_tgt is None:
            raise RuntimeError("belly_track_mm needs pin targets (a muscleToBonePin or belly_attach block)")
        goal = self._to_user(self._pin_tgt)
        pos = self.positions_np()
        idx = self._cons_pts if self.target_mode == "points" else slice(None)
        d = np.linalg.norm(pos[idx] - goal[idx], axis=1)
        return float(np.percentile(d, 50) * 1e3), float(d.mean() * 1e3)

    def tet_mask_for_muscles(self, names) -> np.ndarray:
        """tet_mask_for_muscles (mg.py:1083-1096): per-tet mask of the muscles
        whose name contains any of ``names`` (the rest mesh's ``muscle_id``
        strings), in the user's tet order."""
        if isinstance(names, str):
            names = [names]
        strings = list(self.scene.meta.get("muscle_names") or [])
        if not strings:
            raise ValueError("the rest mesh has no 'muscle_id' prim attribute names")
        sel = [i for i, m in enumerate(strings) if any(n in m for n in names)]
        return np.isin(self.scene.tet_part, sel)

    def preload_targets(self, frames=None) -> None:
        """preload_targets (mg.py:1216-1231): read every frame's targets once
        (the cons frames of target_mode="points"; the other modes compute theirs
        on the device and have nothing to read)."""
        if self.target_mode != "points":
            return
        if frames is None:
            frames = range(self.start_frame, self.end_frame + 1)
        for f in frames:
            self._cons_targets(int(f))

    def substep_at_frac_frame(self, t: float) -> None:
        """substep_at_frac_frame (mg.py:1421-1432): the kinematic step at the
        fractional frame t (bone targets sampled on the bones' path), then one
        substep of the phase program."""
        self._check_status()
        self._kinematic_step(t)
        self.substep()
        self._post_status()

    def apply_pintotarget_all(self) -> None:
        """Soft pin (apply_pintotarget_all, mg/mg.py:1386-1397): every constraint
        point moves by presubframe_pintotarget x (target - pos) toward its pin
        target (target_pos + rest_offset); a no-op when the factor is <= 0.  The
        constraint points are all vertices, or the cons file's points when
        target_mode="points"."""
        b = self.presubframe_pintotarget
        if b <= 0.0 or self._pin_tgt is None:
            return
        idx = getattr(self, "_presub_idx", None)
        n = self.n_verts if idx is None else int(idx.shape[0])
        capi.check(self._lib.xpbd_blend_to_target(n, C.c_void_p(idx.data_ptr()) if idx is not None else None,
                                                  self.n_verts, C.c_void_p(self._pos4.data_ptr()),
                                                  C.c_void_p(self._pin_tgt.data_ptr()), C.c_float(b), self._sp))

    def _vstep_sdf_only(self, coll) -> None:
        sdf = coll.struct()
        capi.check(self._lib.xpbd_vertex_step(C.byref(self._prm), C.byref(self._verts), capi.OP_SDF, C.byref(sdf),
                                              self._sp))

    def build_program(self):
        """mg.py:1322-1378: pre_phase, iter_phase, post_phase."""
        s = self

        def pre_phase():
            s.integrate()
            if s.use_multigrid:
                s._multigrid_pre()
            s.apply_pintotarget()

        def iter_phase():
            for it in range(s.fine_iters):
                s.clear()
                s.solve_constraints(run_extras=False)
                s.apply_dP()
                s._solve_m2m_glue()
                s.apply_pintotarget()
                for fn in getattr(s, "collision_solvers_iter", None) or []:
                    fn(it)

        def post_phase():
            if s.fascia is not None:
                s.fascia.substep()
            for fn in getattr(s, "collision_solvers", None) or []:
                fn()
            s.update_velocities()

        self.program = [pre_phase, iter_phase, post_phase]

    def substep(self) -> None:
        if getattr(self, "program", None) is None:
            self.build_program()
        for phase in self.program:
            phase()

    def _multigrid_pre(self) -> None:
        """_hpbd_vcycle (mg.py:1064-1079); the fine re-pin follows in pre_phase."""
        self.mg.vcycle(pin_fine=False)

    def _kinematic_step(self, t: float) -> None:
        """mg.py:1399-1407: targets for frame t, hard pin, soft pin of all points."""
        if self._frame_loaded != t:
            self.load_frame_targets(t)
        self._targets_kernel()
        if self.mg is not None:
            self.mg.refresh_target()
        if getattr(self, "bone_collider", None) is not None:
            self.bone_collider.bake()
        self.apply_pintotarget()
        self.apply_pintotarget_all()

    def _fusable(self) -> bool:
        cs = getattr(self, "collision_solvers", None) or []
        its = getattr(self, "collision_solvers_iter", None) or []
        dcd = getattr(self, "dcd", None)
        return (all(dcd is not None and fn == dcd.solve for fn in its) and not getattr(self, "constraint_solvers", None)
                and all(getattr(c, "graph_safe", False) for c in cs) and len(cs) <= 1
                and getattr(self, "program", None) is None and not getattr(self, "use_sliding", False))

    def _frame_fused(self) -> None:
        self._targets_kernel()
        if self.fascia is not None:
            self.fascia.advect()  # step_frame (mg.py:1413-1416): once per frame, before the substeps
        if self.mg is not None:
            self.mg.refresh_target()
        sdf = self.collision_solvers[0] if self.collision_solvers else None
        if sdf is not None:
            sdf.bake()
        self._sdf = sdf
        pin = capi.OP_PIN if self._has_pins else 0
        if pin:
            self._vstep(capi.OP_PIN)
        self.apply_pintotarget_all()
        vel = 0 if self.quasi_static else capi.OP_VELOCITY
        push = capi.OP_SDF if sdf is not None else 0
        for sub in range(self.nsubsteps):
            if self.mg is None:
                self._vstep(capi.OP_PREDICT | pin | ((push | vel) if sub > 0 else 0))
            else:
                self._vstep(capi.OP_PREDICT | ((push | vel) if sub > 0 else 0))
                self.mg.vcycle(pin_fine=bool(pin))
            self._substep_iterations()
            if self.fascia is not None:  # post_phase (mg.py:1361-1364), before the push-out and velocity
                self.fascia.substep()
        if push | vel:
            self._vstep(push | vel)

    def _substep_iterations(self) -> None:
        """The fine iterations of one substep in the fused frame: the persistent
        pass when no hook runs between iterations, else one iteration at a time
        (the primitive order when the muscle-to-muscle glue is on)."""
        if self.n_m2m:
            for it in range(self.fine_iters):
                self._m2m_iteration()
                for fn in self.collision_solvers_iter:
                    fn(it)
            return
        if not self.collision_solvers_iter:
            self._fused_iterations(self.fine_iters)
            return
        for it in range(self.fine_iters):
            self._hook_iteration()
            for fn in self.collision_solvers_iter:
                fn(it)

    def _hook_iteration(self) -> None:
        """One fused iteration before a hook: a one-iteration persistent launch
        (one kernel, vertices staged once) when the tiles fit and
        ``persistent_between_hooks`` is set, else the per-iteration tile pass
        and boundary launch."""
        if self.persistent_between_hooks:
            self._fused_iterations(1)
        else:
            self._fused_iteration()

    def step_frame(self, frame: int) -> None:
        """mg.py:1409-1418: kinematic step then nsubsteps substeps at that pose.
        Raises if an earlier frame's status word (checked without waiting)
        shows a barrier timeout or an accumulator overflow."""
        self._check_status()
        if self._frame_loaded != frame:
            self.load_frame_targets(frame)
        if self._fusable():
            self._graph("frame", self._frame_fused)
        else:
            self._kinematic_step(frame)
            if self.fascia is not None:
                self.fascia.advect()
            for _ in range(self.nsubsteps):
                self.substep()
        self._post_status()
        self.step_cnt += 1
