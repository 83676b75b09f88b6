"""Learned coarse warm start for the multigrid cage.

Per substep, after the inertial prediction x_pred of the fine mesh:

  1. restrict x_pred to the cage: c_pred (the previous substep's cage state
     c_prev is the prior of the regularised Galerkin restriction);
  2. 64 features per cage vertex (xpbd_cage_features);
  3. the MLP (CageMLP: tensor-core GEMMs) predicts the cage correction
     dc = c* - c_pred in mm, where c* is the restriction of a converged fine
     solve (200 plain Jacobi iterations from x_pred);
  4. the fine warm start x_ws = x_pred + P dc (delta prolongation, pins
     re-applied);
  5. fallback (judged on the cage, before 4): if the corrected cage's ARAP
     residual exceeds the predicted cage's, the correction is dropped and the
     solve starts from x_pred (xpbd_fallback_select: a device-side choice, no
     host sync);
  6. N plain fine Jacobi iterations (the persistent pass);
  7. restrict the result to the cage: the next substep's c_prev.

With ``fallback="residual"`` the fallback is the plain solver itself: the
substep also runs N plain iterations from x_pred, and the learned result is
replaced by the plain one whenever its post-iteration fine ARAP residual
exceeds the plain solver's (a device-side choice).  That is the rule as
stated for the learned form, at the price of the plain solve on every
substep; the cage rule above is its cheap stand-in.

The training data are the plain solver's own trajectories: for seeds of bone
motion and fiber activation, each substep's features and its converged cage
correction, generated and kept on the GPU; training runs the library's
forward, backward and Adam kernels.  ``python -m rlmusclev2_b200.learned``
runs data generation, training and the held-out evaluation and writes the
weights and a JSON report.
"""
from __future__ import annotations

import argparse
import copy
import ctypes as C
import json
import math
import time
from pathlib import Path

import numpy as np
import torch

from . import _capi as capi
from .cagenet import CageMLP
from .meshgen import reseed_motion
from .mg import MultiGridSim, load_config

PKG = Path(__file__).resolve().parent
CONFIG = PKG / "configs" / "humanv2_synth_mg_dcd.json"
WEIGHTS = PKG / "weights" / "cage_mlp_humanv2.npz"
SCALE_MM = 1000.0


def learned_config() -> dict:
    """Config 3's mesh, cage and constraint set (ARAP, SNH fascia, fiber,
    belly attach, tendon pins, SDF push-out) without the triangle DCD, whose
    contacts would run inside every one of the converged solve's iterations."""
    cfg = load_config(str(CONFIG))
    cfg = copy.deepcopy(cfg)
    (cfg.get("demo") or {}).pop("self_collision", None)
    cfg["use_multigrid"] = True
    return cfg


def _cage_static(sim: MultiGridSim):
    return cage_static(sim.mg.cage, sim.scene)


def cage_static(cage, sc):
    """Host-side cage description: owner muscle, the six lattice neighbours in
    the owner's frame, end bones and axial weight, 24 static features (rest
    position in the muscle frame, fiber axis, 3 x 3 x 2 Fourier terms)."""
    p = cage.coarse_pos.astype(np.float64)
    nc = p.shape[0]
    _, owner = np.unique(cage.blk_base, return_inverse=True)
    owner = owner.astype(np.int64)
    R = sc.muscle_rot[owner]
    cen = sc.muscle_center[owner]
    L = sc.muscle_len[owner]
    u = np.einsum("nij,ni->nj", R, p - cen) / L[:, None]
    # lattice neighbours from the cage tets' edges, classified in the owner's frame
    t = cage.coarse_tet.astype(np.int64)
    e = np.concatenate([t[:, [a, b]] for a in range(4) for b in range(4) if a != b])
    e = np.unique(e, axis=0)
    # the lattice spacing is the shortest edge (the 6-tet split adds face and body diagonals)
    spacing = float(np.percentile(np.linalg.norm(p[e[:, 1]] - p[e[:, 0]], axis=1), 5))
    d = np.einsum("nij,ni->nj", R[e[:, 0]], p[e[:, 1]] - p[e[:, 0]]) / spacing
    nbr = np.full((nc, 6), -1, np.int64)
    for ax in range(3):
        others = [k for k in range(3) if k != ax]
        straight = (np.abs(d[:, others]).max(1) < 0.1) & (np.abs(np.abs(d[:, ax]) - 1.0) < 0.1)
        for sgn, slot in ((1.0, 2 * ax), (-1.0, 2 * ax + 1)):
            sel = straight & (np.sign(d[:, ax]) == sgn)
            nbr[e[sel, 0], slot] = e[sel, 1]
    # end bones of each muscle (all its fine vertices share them) and the axial weight
    nm = sc.muscle_rot.shape[0]
    ends = np.zeros((nm, 2), np.int64)
    for m in range(nm):
        v = np.nonzero(sc.vert_part == m)[0]
        ends[m] = sc.vert_bone[v[0]]
    cbone = ends[owner].astype(np.int32)
    cw = np.clip(u[:, 0] + 0.5, 0.0, 1.0).astype(np.float32)
    four = []
    for f in range(3):
        for k in range(3):
            four += [np.sin(np.pi * 2 ** f * u[:, k]), np.cos(np.pi * 2 ** f * u[:, k])]
    stat = np.concatenate([u, R[:, :, 0], np.stack(four, 1)], 1).astype(np.float32)
    assert stat.shape[1] == 24
    return dict(owner=owner.astype(np.int32), nbr=nbr.astype(np.int32), cbone=cbone, cw=cw, stat=stat,
                n_muscles=nm)


def bone_relative(sc, frame: int) -> np.ndarray:
    """(n_bones, 12) [R | t] of T(frame) T(frame - 1)^-1, row-major."""
    Ta, Tb = sc.bone_transforms(frame), sc.bone_transforms(frame - 1)
    Rr = np.einsum("bij,bkj->bik", Ta[:, :, :3], Tb[:, :, :3])
    tr = Ta[:, :, 3] - np.einsum("bij,bj->bi", Rr, Tb[:, :, 3])
    return np.concatenate([Rr, tr[:, :, None]], 2).reshape(-1, 12).astype(np.float32)


class LearnedWarmStart:
    """Substep driver of the plain and the learned forms on one MultiGridSim
    (config 3's mesh and cage); see the module docstring."""

    def __init__(self, sim: MultiGridSim, net: CageMLP | None = None):
        if sim.mg is None:
            raise ValueError("the learned warm start needs the multigrid cage (use_multigrid)")
        self.sim, self.mg = sim, sim.mg
        self.lib = sim._lib
        self.sp = sim._sp
        dev = sim.device
        st = _cage_static(sim)
        self.nc = int(st["owner"].shape[0])
        self.net = net if net is not None else CageMLP(dev, self.nc, stream=sim._stream)
        T = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dt)  # noqa: E731
        self._owner, self._nbr = T(st["owner"]), T(st["nbr"])
        self._cbone, self._cw, self._stat = T(st["cbone"]), T(st["cw"]), T(st["stat"])
        self._act = torch.zeros(st["n_muscles"], dtype=torch.float32, device=dev)
        self._bone_rel = torch.zeros((sim.scene.n_bones, 12), dtype=torch.float32, device=dev)
        self._bone_rel_host = torch.zeros((sim.scene.n_bones, 12), dtype=torch.float32).pin_memory()
        self._act_host = torch.zeros(st["n_muscles"], dtype=torch.float32).pin_memory()
        self._lib_d = self.mg._t["coarse_lib"]
        cf = capi.XpbdCageFeatures()
        cf.n_cage, cf.m_pad = self.nc, self.net.m_pad
        cf.coarse_lib, cf.nbr, cf.owner = self._lib_d.data_ptr(), self._nbr.data_ptr(), self._owner.data_ptr()
        cf.act_muscle, cf.cage_bone, cf.cage_w = self._act.data_ptr(), self._cbone.data_ptr(), self._cw.data_ptr()
        cf.bone_rel, cf.stat = self._bone_rel.data_ptr(), self._stat.data_ptr()
        self._cf = cf
        co = self.mg.coarse
        self._c0 = co._pos4.clone()
        cf.c_rest4, cf.c_target4 = self._c0.data_ptr(), self.mg.pin4.data_ptr()
        self._norm = torch.zeros((64, 2), dtype=torch.float32, device=dev)
        cf.norm = self._norm.data_ptr()
        self.set_norm(None)
        self._cprev = torch.zeros_like(co._pos4)
        self._saved = torch.zeros_like(sim._pos4)
        self._saved_plain = torch.zeros_like(sim._pos4)
        self._mbuf = torch.zeros((2, 8), dtype=torch.float64, device=dev)
        self.fallbacks = torch.zeros(1, dtype=torch.int32, device=dev)
        self.plain_taken = torch.zeros(1, dtype=torch.int32, device=dev)  # residual-rule fallbacks
        self.target = torch.zeros((self.nc, 3), dtype=torch.float32, device=dev)
        cfg = sim.cfg
        coll = (cfg.get("demo") or {}).get("collision") or {}
        self.push = capi.OP_SDF if coll.get("enabled", False) else 0
        self.vel = 0 if sim.quasi_static else capi.OP_VELOCITY
        self.pin = capi.OP_PIN if sim._has_pins else 0
        # the correction is dropped when it more than doubles the cage's ARAP
        # residual: pulling the cage toward its bone targets raises that
        # residual a little even for a good correction
        self.fallback_factor = 2.0

    def set_norm(self, norm: np.ndarray | None, y_scale: float = 1.0) -> None:
        """Feature standardisation ((64, 2): mean, 1/std; None = identity) and
        the network output's scale in mm."""
        n = np.zeros((64, 2), np.float32)
        n[:, 1] = 1.0
        if norm is not None:
            n[:] = norm
        with torch.cuda.stream(self.sim._stream):
            self._norm.copy_(torch.from_numpy(n).to(self.sim.device))
        self.sim.synchronize()
        self.norm_np = n
        self.y_scale = float(y_scale)

    # ------------------------------------------------------------- state
    def reset(self, scene) -> None:
        """Rest state, the motion and activation schedule of ``scene``."""
        sim = self.sim
        sim.scene = scene
        sim.set_positions(scene.verts, also_prev=True)
        sim.set_velocities(np.zeros_like(scene.verts))
        with torch.cuda.stream(sim._stream):
            self.mg.coarse._pos4.copy_(self._c0)
        sim._frame_loaded = None
        sim.synchronize()

    def begin_frame(self, frame: int) -> None:
        """Frame inputs (bone poses, activation, bone-relative motion for the
        features), bone targets, SDF bake and the frame's first pin."""
        sim, sc = self.sim, self.sim.scene
        sim.set_fiber_activation(sc.activation(frame))
        sim.load_frame_targets(frame)
        sim._targets_kernel()
        self.mg.refresh_target()  # restricted bone-driven targets (a feature)
        self._h_sync()
        self._bone_rel_host.numpy()[:] = bone_relative(sc, frame)
        self._act_host.numpy()[:] = sc.muscle_activation(frame)
        with torch.cuda.stream(sim._stream):
            self._bone_rel.copy_(self._bone_rel_host, non_blocking=True)
            self._act.copy_(self._act_host, non_blocking=True)
        self._ev = torch.cuda.Event()
        self._ev.record(sim._stream)
        coll = sim.collision_solvers[0] if sim.collision_solvers else None
        if coll is not None:
            coll.bake()
        sim._sdf = coll
        if self.pin:
            sim._vstep(capi.OP_PIN)

    def _h_sync(self):
        ev = getattr(self, "_ev", None)
        if ev is not None:
            ev.synchronize()

    def end_frame(self) -> None:
        if self.push | self.vel:
            self.sim._vstep(self.push | self.vel)

    def predict(self, sub: int) -> None:
        """Inertial prediction (with the previous substep's push-out and velocity
        update), then c_prev <- cage state, c_pred <- restrict(x_pred)."""
        sim, mg = self.sim, self.mg
        sim._vstep(capi.OP_PREDICT | self.pin | ((self.push | self.vel) if sub > 0 else 0))
        with torch.cuda.stream(sim._stream):
            self._cprev.copy_(mg.coarse._pos4)
        capi.check(self.lib.xpbd_mg_restrict(C.byref(mg.g), C.c_void_p(sim._pos4.data_ptr()),
                                             C.c_void_p(mg.coarse._pos4.data_ptr()), C.c_void_p(mg.prev.data_ptr()),
                                             None, self.sp))

    def features(self) -> None:
        net = self.net
        capi.check(self.lib.xpbd_cage_features(C.byref(self._cf), C.c_void_p(self.mg.prev.data_ptr()),
                                               C.c_void_p(self._cprev.data_ptr()), C.c_void_p(net.X.data_ptr()),
                                               C.c_void_p(net.Xt.data_ptr()), self.sp))

    def _metrics_into(self, k: int) -> None:
        sim = self.sim
        capi.check(self.lib.xpbd_metrics(C.byref(sim._tiles), C.byref(sim._verts),
                                         C.c_void_p(self._mbuf[k].data_ptr()), self.sp))

    def _coarse_metrics_into(self, k: int) -> None:
        co = self.mg.coarse
        capi.check(self.lib.xpbd_metrics(C.byref(co._tiles), C.byref(co._verts),
                                         C.c_void_p(self._mbuf[k].data_ptr()), self.sp))

    def warm_start(self, fallback: bool = True) -> None:
        """Network forward, cage correction, fallback, delta prolongation (+ fine
        pins).  The fallback is judged on the cage: if the corrected cage's ARAP
        residual (against the cage's rest) exceeds the predicted cage's, the
        correction is dropped (a device-side choice) and x_pred stays."""
        sim, mg, net = self.sim, self.mg, self.net
        if fallback:
            self._coarse_metrics_into(0)
        net.forward(self.nc, train=False)
        capi.check(self.lib.xpbd_cage_apply(self.nc, C.c_void_p(self._lib_d.data_ptr()),
                                            C.c_void_p(mg.prev.data_ptr()), C.c_void_p(net.Y.data_ptr()),
                                            net.Y.shape[1], C.c_float(self.y_scale / SCALE_MM),
                                            C.c_void_p(mg.coarse._pos4.data_ptr()), self.sp))
        if fallback:
            self._coarse_metrics_into(1)
            capi.check(self.lib.xpbd_fallback_select(mg.coarse.n_verts, C.c_void_p(self._mbuf[1].data_ptr()),
                                                     C.c_void_p(self._mbuf[0].data_ptr()),
                                                     C.c_float(self.fallback_factor),
                                                     C.c_void_p(mg.prev.data_ptr()),
                                                     C.c_void_p(mg.coarse._pos4.data_ptr()),
                                                     C.c_void_p(self.fallbacks.data_ptr()), self.sp))
        vf = sim._vflags.data_ptr() if (self.pin and sim._vflags is not None) else None
        pt = sim._pin_tgt.data_ptr() if (self.pin and sim._pin_tgt is not None) else None
        capi.check(self.lib.xpbd_mg_prolong_delta(C.byref(mg.g), C.c_void_p(mg.coarse._pos4.data_ptr()),
                                                  C.c_void_p(mg.prev.data_ptr()), C.c_void_p(sim._pos4.data_ptr()),
                                                  C.c_void_p(vf) if vf else None, C.c_void_p(pt) if pt else None,
                                                  self.sp))

    def ideal_warm_start(self) -> None:
        """The warm start a perfect network would give: the cage moved by the
        substep's true correction (``self.target``, from target_from_state),
        prolongated onto the fine mesh (+ fine pins).  An evaluation device: it
        bounds what any cage correction can do for the iterations after it."""
        sim, mg = self.sim, self.mg
        capi.check(self.lib.xpbd_cage_apply(self.nc, C.c_void_p(self._lib_d.data_ptr()),
                                            C.c_void_p(mg.prev.data_ptr()), C.c_void_p(self.target.data_ptr()), 3,
                                            C.c_float(1.0 / SCALE_MM), C.c_void_p(mg.coarse._pos4.data_ptr()),
                                            self.sp))
        vf = sim._vflags.data_ptr() if (self.pin and sim._vflags is not None) else None
        pt = sim._pin_tgt.data_ptr() if (self.pin and sim._pin_tgt is not None) else None
        capi.check(self.lib.xpbd_mg_prolong_delta(C.byref(mg.g), C.c_void_p(mg.coarse._pos4.data_ptr()),
                                                  C.c_void_p(mg.prev.data_ptr()), C.c_void_p(sim._pos4.data_ptr()),
                                                  C.c_void_p(vf) if vf else None, C.c_void_p(pt) if pt else None,
                                                  self.sp))

    def iterate(self, n: int) -> None:
        self.sim._fused_iterations(n)

    def restrict_final(self) -> None:
        """Cage state <- restrict(final fine state) (prior: the current cage)."""
        sim, mg = self.sim, self.mg
        capi.check(self.lib.xpbd_mg_restrict(C.byref(mg.g), C.c_void_p(sim._pos4.data_ptr()),
                                             C.c_void_p(mg.coarse._pos4.data_ptr()), None, None, self.sp))

    def target_from_state(self) -> None:
        """target = (restrict(current fine state) - c_pred) in mm (cage order);
        leaves the restricted state as the cage state."""
        mg = self.mg
        with torch.cuda.stream(self.sim._stream):
            mg.coarse._pos4.copy_(mg.prev)
        self.restrict_final()
        capi.check(self.lib.xpbd_cage_target(self.nc, C.c_void_p(self._lib_d.data_ptr()),
                                             C.c_void_p(mg.coarse._pos4.data_ptr()), C.c_void_p(mg.prev.data_ptr()),
                                             C.c_float(SCALE_MM), C.c_void_p(self.target.data_ptr()), self.sp))

    # ------------------------------------------------------- one substep
    def substep(self, sub: int, n_iters: int, learned: bool, fallback=True) -> None:
        """One substep of the learned form, or of the plain form (prediction and
        iterations only: the plain solver needs no cage).  ``fallback``: True
        the cage rule, False none, "residual" the plain solver's residual."""
        if not learned:
            self.sim._vstep(capi.OP_PREDICT | self.pin | ((self.push | self.vel) if sub > 0 else 0))
            self.iterate(n_iters)
            return
        self.predict(sub)
        if fallback == "residual":
            self.plain_checked(n_iters)
        else:
            self.features()
            self.warm_start(bool(fallback))
            self.iterate(n_iters)
        self.restrict_final()

    def plain_checked(self, n_iters: int) -> None:
        """From x_pred (after predict): the plain solve (n_iters iterations,
        its fine metrics and result kept), then the learned solve from the same
        x_pred; the plain result replaces the learned one when the learned
        post-iteration ARAP residual exceeds the plain one or is not finite
        (xpbd_fallback_select, counted in ``plain_taken``)."""
        sim = self.sim
        with torch.cuda.stream(sim._stream):
            self._saved.copy_(sim._pos4)
        self.iterate(n_iters)
        self._metrics_into(1)
        with torch.cuda.stream(sim._stream):
            self._saved_plain.copy_(sim._pos4)
            sim._pos4.copy_(self._saved)
        self.features()
        self.warm_start(fallback=False)
        self.iterate(n_iters)
        self._metrics_into(0)
        capi.check(self.lib.xpbd_fallback_select(sim.n_verts, C.c_void_p(self._mbuf[0].data_ptr()),
                                                 C.c_void_p(self._mbuf[1].data_ptr()), C.c_float(1.0),
                                                 C.c_void_p(self._saved_plain.data_ptr()),
                                                 C.c_void_p(sim._pos4.data_ptr()),
                                                 C.c_void_p(self.plain_taken.data_ptr()), self.sp))

    def frame(self, frame: int, n_iters: int, learned: bool, fallback=True) -> None:
        self.begin_frame(frame)
        for sub in range(self.sim.nsubsteps):
            self.substep(sub, n_iters, learned, fallback)
        self.end_frame()


# ---------------------------------------------------------------------------
# data, training, evaluation


def generate(ws: LearnedWarmStart, seeds, frames: int, conv_iters: int = 200, log=print):
    """Converged trajectories of the plain solver: per substep the features
    (BF16, cage rows) and the converged cage correction (mm)."""
    sim, net = ws.sim, ws.net
    S = len(seeds) * frames * sim.nsubsteps
    X = torch.zeros((S, ws.nc, 64), dtype=torch.bfloat16, device=sim.device)
    Y = torch.zeros((S, ws.nc, 3), dtype=torch.float32, device=sim.device)
    base = sim.scene
    k = 0
    t0 = time.time()
    for si, seed in enumerate(seeds):
        ws.reset(reseed_motion(base, seed))
        for f in range(1, frames + 1):
            ws.begin_frame(f)
            for sub in range(sim.nsubsteps):
                ws.predict(sub)
                ws.features()
                ws.iterate(conv_iters)
                ws.target_from_state()
                with torch.cuda.stream(sim._stream):
                    X[k].copy_(net.X[:ws.nc])
                    Y[k].copy_(ws.target)
                k += 1
            ws.end_frame()
        sim.synchronize()
        log(f"  seed {seed}: {k} substeps, {time.time() - t0:.1f} s")
    ws.reset(base)
    return X, Y


def standardise(X, Y):
    """Per-feature mean and 1/std of the raw features and the targets' rms;
    X and Y are standardised in place.  Returns (norm (64, 2), y_scale)."""
    Xf = X.view(-1, 64)
    mu = torch.zeros(64, dtype=torch.float64, device=X.device)
    sq = torch.zeros(64, dtype=torch.float64, device=X.device)
    n = Xf.shape[0]
    for a in range(0, n, 1 << 22):
        blk = Xf[a:a + (1 << 22)].double()
        mu += blk.sum(0)
        sq += (blk * blk).sum(0)
    mu /= n
    std = (sq / n - mu * mu).clamp_min(1e-12).sqrt()
    inv = torch.where(std > 1e-6, 1.0 / std, torch.zeros_like(std))
    for a in range(0, n, 1 << 22):
        blk = Xf[a:a + (1 << 22)]
        blk.copy_(((blk.double() - mu) * inv).to(torch.bfloat16))
    ys = float(Y.double().pow(2).mean().sqrt().item())
    Y /= ys
    norm = torch.stack([mu, inv], 1).float().cpu().numpy()
    return norm, ys


def train(net: CageMLP, X, Y, steps: int, lr: float = 1e-3, seed: int = 0, log=print):
    """Adam on one substep's cage (all vertices) per step, cosine-decayed lr."""
    rng = np.random.default_rng(seed)
    S, nc = X.shape[0], X.shape[1]
    hist = []
    with torch.cuda.stream(net.stream):
        net.loss.zero_()
    acc = 0
    for it in range(steps):
        s = int(rng.integers(S))
        with torch.cuda.stream(net.stream):
            net.X[:nc].copy_(X[s])
            net.Xt[:, :nc].copy_(X[s].t())
        net.forward(nc)
        net.backward(nc, Y[s])
        net.adam_step(lr=lr * 0.5 * (1.0 + math.cos(math.pi * it / steps)))
        acc += 1
        if (it + 1) % max(1, steps // 20) == 0 or it == steps - 1:
            net.stream.synchronize()
            hist.append((it + 1, float(net.loss.item()) / (acc * nc * 3)))
            log(f"  step {it + 1}: mse {hist[-1][1]:.4f} (standardised)")
            with torch.cuda.stream(net.stream):
                net.loss.zero_()
            acc = 0
    return hist


def evaluate(ws: LearnedWarmStart, seeds, frames: int, ns, conv_iters: int = 200, log=print, ideal: bool = False,
             checked_ns=()):
    """Max fine-vertex error (mm) against the converged solve from the same
    prediction, for the plain form and the learned form after n iterations
    (n in ns), on every substep of the held-out trajectories (which follow
    the converged solve).  With ``ideal``, also the form warm-started by the
    substep's true cage correction (what a perfect network would give); for
    n in ``checked_ns`` the learned form checked against the plain solver's
    residual (``fallback="residual"``, form "checked")."""
    sim = ws.sim
    base = sim.scene
    ns = sorted(ns)
    forms = ("plain", "learned", "learned_raw") + (("ideal",) if ideal else ())
    err = {f: {n: [] for n in ns} for f in forms}
    rms = {f: {n: [] for n in ns} for f in forms}
    if checked_ns:
        err["checked"] = {n: [] for n in checked_ns}
        rms["checked"] = {n: [] for n in checked_ns}
    xpred = torch.zeros_like(sim._pos4)
    cpred = torch.zeros_like(ws.mg.coarse._pos4)
    cstar = torch.zeros_like(ws.mg.coarse._pos4)
    for seed in seeds:
        ws.reset(reseed_motion(base, seed))
        for f in range(1, frames + 1):
            ws.begin_frame(f)
            for sub in range(sim.nsubsteps):
                ws.predict(sub)
                with torch.cuda.stream(sim._stream):
                    xpred.copy_(sim._pos4)
                    cpred.copy_(ws.mg.coarse._pos4)
                # the converged solve first: its restriction is the true correction
                ws.iterate(conv_iters)
                with torch.cuda.stream(sim._stream):
                    ref = sim._pos4[:, :3].clone()
                    refp = sim._pos4.clone()
                    ws.mg.coarse._pos4.copy_(cpred)
                ws.target_from_state()
                with torch.cuda.stream(sim._stream):
                    cstar.copy_(ws.mg.coarse._pos4)
                for form in forms:
                    with torch.cuda.stream(sim._stream):
                        sim._pos4.copy_(xpred)
                        ws.mg.coarse._pos4.copy_(cpred)
                    if form == "ideal":
                        ws.ideal_warm_start()
                    elif form != "plain":
                        ws.features()
                        ws.warm_start(fallback=(form == "learned"))
                    done = 0
                    for n in ns:
                        ws.iterate(n - done)
                        done = n
                        with torch.cuda.stream(sim._stream):
                            d = (sim._pos4[:, :3] - ref).norm(dim=1)
                            err[form][n].append(d.max())
                            rms[form][n].append(d.pow(2).mean().sqrt())
                for n in checked_ns:
                    with torch.cuda.stream(sim._stream):
                        sim._pos4.copy_(xpred)
                        ws.mg.coarse._pos4.copy_(cpred)
                    ws.plain_checked(n)
                    with torch.cuda.stream(sim._stream):
                        d = (sim._pos4[:, :3] - ref).norm(dim=1)
                        err["checked"][n].append(d.max())
                        rms["checked"][n].append(d.pow(2).mean().sqrt())
                # the trajectory follows the converged solve
                with torch.cuda.stream(sim._stream):
                    sim._pos4.copy_(refp)
                    ws.mg.coarse._pos4.copy_(cstar)
            ws.end_frame()
        log(f"  eval seed {seed} done")
    sim.synchronize()
    ws.reset(base)
    cv = lambda e: {form: {n: (torch.stack(v) * SCALE_MM).cpu().numpy() for n, v in d.items()}  # noqa: E731
                    for form, d in e.items()}
    return cv(err), cv(rms)


def iterations_to(err_by_n: dict, tol_mm: float):
    """Smallest n (log-linear interpolation between the evaluated counts) at
    which the worst substep's max error reaches tol_mm; None if none does."""
    ns = sorted(err_by_n)
    worst = [float(np.max(err_by_n[n])) for n in ns]
    for k, (n, e) in enumerate(zip(ns, worst)):
        if e <= tol_mm:
            if k == 0:
                return float(n)
            n0, e0 = ns[k - 1], worst[k - 1]
            if e <= 0.0:  # the reference itself (n = conv_iters): interpolate linearly
                return float(n0 + (e0 - tol_mm) / e0 * (n - n0))
            t = (math.log(e0) - math.log(tol_mm)) / max(math.log(e0) - math.log(e), 1e-12)
            return float(n0 + t * (n - n0))
    return None


def time_frame(ws: LearnedWarmStart, n_iters: int, learned: bool, frames=(5, 6, 7), fallback: bool = True) -> float:
    """GPU ms per frame of a form (CUDA events on the engine stream)."""
    sim = ws.sim
    s = sim._stream
    ws.frame(4, n_iters, learned, fallback)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = 0.0
    for f in frames:
        ws.begin_frame(f)
        sim.synchronize()
        e0.record(s)
        for sub in range(sim.nsubsteps):
            ws.substep(sub, n_iters, learned, fallback)
        e1.record(s)
        e1.synchronize()
        ws.end_frame()
        tot += e0.elapsed_time(e1)
    return tot / len(frames)


def profile_case(n_iters: int = 20) -> None:
    """Two eager frames of each form (for a kernel launch list)."""
    sim = MultiGridSim(learned_config())
    ws = LearnedWarmStart(sim)
    load_weights(ws)
    ws.reset(reseed_motion(sim.scene, 41))
    for f in (1, 2):
        ws.frame(f, n_iters, learned=False)
    for f in (3, 4):
        ws.frame(f, n_iters, learned=True)
    sim.synchronize()


def save_weights(ws: LearnedWarmStart, path: Path, meta: dict) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    sd = ws.net.state_dict()
    np.savez_compressed(path, meta=np.array(json.dumps(meta)), norm=ws.norm_np, y_scale=np.float32(ws.y_scale), **sd)


def load_weights(ws: LearnedWarmStart, path: Path = WEIGHTS) -> dict:
    d = np.load(path)
    ws.net.load_state_dict({k: d[k] for k in d.files if k[0] in "Wb" and k[1:].isdigit()})
    ws.set_norm(d["norm"], float(d["y_scale"]))
    return json.loads(str(d["meta"])) if "meta" in d.files else {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", default="1-40")
    ap.add_argument("--eval-seeds", default="41-48")
    ap.add_argument("--frames", type=int, default=50)
    ap.add_argument("--eval-frames", type=int, default=4)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--conv-iters", type=int, default=200)
    ap.add_argument("--ns", default="5,10,20,30,40,60,80,100,120,160")
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-only", action="store_true", help="load --out's weights, evaluate and time")
    ap.add_argument("--profile-case", action="store_true", help="two eager frames of each form and exit")
    args = ap.parse_args()
    if args.profile_case:
        profile_case()
        return
    rng = lambda s: list(range(int(s.split("-")[0]), int(s.split("-")[1]) + 1))  # noqa: E731
    t0 = time.time()
    sim = MultiGridSim(learned_config())
    ws = LearnedWarmStart(sim)
    print(f"setup {time.time() - t0:.1f} s: {sim.NT} tets, cage {ws.nc} verts", flush=True)
    if args.eval_only:
        meta0 = load_weights(ws, Path(args.out))
        ys, hist = float(ws.y_scale), []
        print(f"weights {meta0}", flush=True)
    else:
        X, Y = generate(ws, rng(args.train_seeds), args.frames, args.conv_iters, log=lambda m: print(m, flush=True))
        norm, ys = standardise(X, Y)
        ws.set_norm(norm, ys)
        print(f"data: {X.shape[0]} substeps, target rms {ys:.4f} mm", flush=True)
        hist = train(ws.net, X, Y, args.steps, args.lr, log=lambda m: print(m, flush=True))
        del X, Y
        torch.cuda.empty_cache()
    ns = [int(x) for x in args.ns.split(",")]
    ev, ev_rms = evaluate(ws, rng(args.eval_seeds), args.eval_frames, ns, args.conv_iters,
                          log=lambda m: print(m, flush=True))
    summary = {form: {n: dict(max=float(v.max()), p95=float(np.percentile(v, 95)), mean=float(v.mean()),
                              rms_mean=float(ev_rms[form][n].mean()))
                      for n, v in d.items()} for form, d in ev.items()}
    per_frame = {form: {n: [float(x) for x in v.reshape(-1, sim.nsubsteps).max(1)] for n, v in d.items()}
                 for form, d in ev.items()}
    for n in ns:
        print(f"n={n:4d} " + "  ".join(f"{f}: max {summary[f][n]['max']:.4f} p95 {summary[f][n]['p95']:.4f} "
                                       f"rms {summary[f][n]['rms_mean']:.4f}" for f in summary), flush=True)
    timing = {}
    ws.reset(reseed_motion(sim.scene, 41))
    for n in ns:
        timing[n] = dict(plain=time_frame(ws, n, False), learned=time_frame(ws, n, True))
        print(f"n={n:4d} ms/frame plain {timing[n]['plain']:.3f} learned {timing[n]['learned']:.3f}", flush=True)
    meta = dict(train_seeds=args.train_seeds, frames=args.frames, steps=args.steps, conv_iters=args.conv_iters,
                final_mse_standardised=hist[-1][1] if hist else None, target_rms_mm=ys)
    if not args.eval_only:
        save_weights(ws, Path(args.out), meta)
    rep = dict(meta=meta, history=hist, eval=summary, per_frame=per_frame, timing_ms_per_frame=timing,
               fallbacks=int(ws.fallbacks.item()))
    if args.report:
        Path(args.report).write_text(json.dumps(rep, indent=1))
    print(f"done in {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()
