"""Batched instances: many independent box muscles stepped as one packed mesh.

The instances of a ``BatchScene`` share one vertex set and one tet set (CSR
offsets per instance); the tile layout keeps every instance's tets in tiles of
their own, so the persistent tet pass runs runs of whole instances as
closed tile ranges (one cooperative launch per range, each holding at most the
resident CTA slots).  Each instance has its own two capsule bones, its own
64^3 SDF grid and its own activation schedule; a frame (bone targets, the
batched SDF bake, 10 substeps) replays as one captured CUDA graph.

``autotune()`` times the tet-pass configurations on the live batch (tile size,
CTAs per SM, persistent ranges vs per-iteration launches, tet-stream prefetch)
and keeps the fastest; results are cached per (GPU, mesh, material set) in a
JSON file.
"""
from __future__ import annotations

import copy
import ctypes as C
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _capi as capi
from .collision import BatchedSdfCollider
from .meshgen import BatchScene, batch_subset, shard_instances
from .mg import MultiGridSim, scene_from_cfg

TUNE_CACHE = Path(os.environ.get("RLMUSCLEV2_B200_TUNE_CACHE", Path(__file__).resolve().parent / "tune_cache.json"))


class BatchSim(MultiGridSim):
    """MultiGridSim over a BatchScene (config keys as MultiGridSim's; the
    collision grid is per instance at the scene's sdf_res)."""

    def __init__(self, cfg: dict, device: str | None = "cuda:0", scene: BatchScene | None = None,
                 shard: tuple[int, int] | None = None):
        cfg = copy.deepcopy(cfg)
        coll = dict((cfg.get("demo") or {}).get("collision") or {})
        cfg.setdefault("demo", {})["collision"] = dict(coll, enabled=False)
        sc = scene if scene is not None else scene_from_cfg(cfg)
        if not isinstance(sc, BatchScene):
            raise TypeError("BatchSim needs a BatchScene (synthetic kind 'batched_boxes')")
        self.instances = np.arange(sc.n_inst)
        if shard is not None:
            rank, world = shard
            self.instances = np.asarray(shard_instances(np.diff(sc.inst_tptr), world)[rank], np.int64)
            sc = batch_subset(sc, self.instances)
        super().__init__(cfg, device, sc)
        self.n_inst = sc.n_inst
        if coll.get("enabled", False):
            self.bone_collider = BatchedSdfCollider(self, sc, contact_offset=float(coll.get("contact_offset", 0.0)),
                                                    max_push=float(coll.get("max_push", -1.0)))
            self.bone_collider.transforms = self._bone_tr
            self.collision_solvers.append(self.bone_collider)
        dev = self.device
        self._inst_act = torch.zeros(self.n_inst, dtype=torch.float32, device=dev)
        self._inst_act_host = torch.zeros(self.n_inst, dtype=torch.float32).pin_memory()
        self._tet_inst_lib = torch.from_numpy(np.ascontiguousarray(sc.tet_inst[self.layout.tet_perm], np.int32)).to(dev)

    # ------------------------------------------------------------ per frame
    def _vstep(self, ops: int) -> None:
        sdf = self._sdf if (ops & capi.OP_SDF) else None
        if sdf is None or not isinstance(sdf, BatchedSdfCollider):
            return super()._vstep(ops)
        capi.check(self._lib.xpbd_vertex_step_batched(C.byref(self._prm), C.byref(self._verts), ops,
                                                      C.byref(sdf.struct()), self._sp))

    def _vstep_sdf_only(self, coll) -> None:
        self._sdf = coll
        self._vstep(capi.OP_SDF)

    def set_instance_activation(self, a_inst) -> None:
        """(n_inst,) activations: one pinned H2D copy of n_inst floats, expanded
        to the tets on the device."""
        if self._t_act is None:
            raise RuntimeError("set_instance_activation requires a fiber constraint")
        a = np.asarray(a_inst, np.float32).reshape(-1)
        if a.shape[0] != self.n_inst:
            raise ValueError(f"{a.shape[0]} activations for {self.n_inst} instances")
        self._act_event.synchronize()
        self._inst_act_host.numpy()[:] = a
        with torch.cuda.stream(self._stream):
            self._inst_act.copy_(self._inst_act_host, non_blocking=True)
        self._act_event.record(self._stream)
        capi.check(self._lib.xpbd_gather(self.NT, 1, C.c_void_p(self._tet_inst_lib.data_ptr()),
                                         C.c_void_p(self._inst_act.data_ptr()), 1,
                                         C.c_void_p(self._t_act.data_ptr()), 1, self._sp))

    def step_frame_inputs(self, frame: int) -> None:
        """The frame's inputs from the scene (activation schedule), then the frame."""
        if self._t_act is not None:
            self.set_instance_activation(self.scene.instance_activation(frame))
        self.step_frame(frame)

    # ------------------------------------------------------------- autotune
    def _candidates(self):
        """Persistent ranges without/with tet-stream prefetch; per-iteration
        launches at the default and the flipped CTAs/SM, with the bulk L2
        prefetch of each tile's tet streams (tile_variant bit 5), and with
        that prefetch and the deferred pass for the tets that need the SVD
        (bit 6)."""
        return [dict(persistent=True, variant=0), dict(persistent=True, variant=4),
                dict(persistent=False, variant=0), dict(persistent=False, variant=1),
                dict(persistent=False, variant=32), dict(persistent=False, variant=33),
                dict(persistent=False, variant=96), dict(persistent=False, variant=97)]

    def _time_iterations(self, n_iters: int, reps: int) -> float:
        """ms per Jacobi iteration with the frame's own grouping: ``reps``
        calls of n_iters fused iterations (n_iters = fine_iterations)."""
        s = self._stream
        self._fused_iterations(n_iters)
        s.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            self._fused_iterations(n_iters)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / (reps * n_iters)

    def _tune_key(self) -> str:
        name = torch.cuda.get_device_name(self.device)
        flags = sorted({int(m["flags"]) for m in self.layout.materials})
        cands = len(self._candidates())
        return f"{name}|nv={self.NV}|nt={self.NT}|inst={self.n_inst}|flags={flags}|iters={self.fine_iters}|cands={cands}"

    def autotune(self, use_cache: bool = True) -> dict:
        """Pick the fastest tet-pass configuration for this batch: persistent
        tile ranges (with or without tet-stream prefetch) or per-iteration
        launches, timed on the current state (positions restored after)."""
        key = self._tune_key()
        cache = {}
        if use_cache and TUNE_CACHE.exists():
            try:
                cache = json.loads(TUNE_CACHE.read_text())
            except Exception:
                cache = {}
        if use_cache and key in cache:
            best = cache[key]
        else:
            saved = self._pos4.clone()
            results = []
            for c in self._candidates():
                if c["persistent"] and not self._persist_fits:
                    continue
                self.use_persistent = c["persistent"]
                self._prm.tile_variant = c["variant"]
                ms = self._time_iterations(self.fine_iters, max(3, 40 // self.fine_iters))
                results.append((ms, c))
                with torch.cuda.stream(self._stream):
                    self._pos4.copy_(saved)
            self._stream.synchronize()
            ms, best = min(results, key=lambda r: r[0])
            best = dict(best, ms_per_iteration=ms, tried=[dict(c, ms=m) for m, c in results])
            cache[key] = best
            if use_cache:
                try:
                    TUNE_CACHE.write_text(json.dumps(cache, indent=1))
                except OSError:
                    pass
        self.use_persistent = bool(best["persistent"])
        self._prm.tile_variant = int(best["variant"])
        self.release_graphs()
        self.tuned = best
        return best
