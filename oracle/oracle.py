"""CPU oracle of the XPBD substep -- TEST INFRASTRUCTURE ONLY.

Python composition of the C restatement in xpbd_oracle.c, in the reference's
program order (MuscleSim.build_program, musclesim.py:107-130).  Used by the
test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product never imports it.  Parity is pinned against the
reference's known-answer tests only (see tests/test_oracle_pins.py): the
reference itself needs NVIDIA Warp and cannot run here.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

T_ATTACH = 1650556
T_TETVOLUME = -215389979
T_TETARAPSVD = -92199132
T_TETARAPANISO = -92199133
T_TETSNH = -503462311

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Prec:
    def __init__(self, name):
        assert name in ("f32", "f64")
        self.name = name
        self.dt = np.float32 if name == "f32" else np.float64
        self.ct = C.c_float if name == "f32" else C.c_double

    def fn(self, base):
        return getattr(lib(), f"{base}_{self.name}")

    def arr(self, a, shape=None):
        x = np.ascontiguousarray(np.asarray(a, dtype=self.dt))
        return x if shape is None else x.reshape(shape)


def svd3(F, prec="f64"):
    P = Prec(prec)
    f = P.arr(F, (9,))
    U, s, V = np.zeros(9, P.dt), np.zeros(3, P.dt), np.zeros(9, P.dt)
    P.fn("orc_svd3")(_p(f), _p(U), _p(s), _p(V))
    return U.reshape(3, 3), s, V.reshape(3, 3)


def precompute_rest(pos0, tets, density, prec="f32"):
    """precompute_rest_kernel (engine.py:199-224): rest_volume, B, mass, total."""
    P = Prec(prec)
    pos0 = P.arr(pos0)
    tets = np.ascontiguousarray(tets, np.int32)
    nt = tets.shape[0]
    rv, B, mass, tot = np.zeros(nt, P.dt), np.zeros((nt, 9), P.dt), np.zeros(pos0.shape[0], P.dt), np.zeros(1, P.dt)
    f = P.fn("orc_precompute_rest")
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, P.ct, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f(nt, _p(pos0), _p(tets), P.ct(density), _p(rv), _p(B), _p(mass), _p(tot))
    return rv, B.reshape(nt, 3, 3), mass, float(tot[0])


def signed_rest_volume(pos0, tets):
    """builder.py:28-43: V0 = det(Dm)/6 of float32 differences (signed), valid mask."""
    tp = np.asarray(pos0, np.float32)[tets]
    cols = (tp[:, :3, :] - tp[:, 3:4, :]).astype(np.float64)
    det = np.linalg.det(np.transpose(cols, (0, 2, 1)))
    return (det / 6.0).astype(np.float32), np.abs(det) > 1e-30


class Table:
    """Reference struct-of-arrays constraint table (engine.py:1179-1211)."""

    def __init__(self):
        self.cols = {k: [] for k in ("type", "pts", "k", "damp", "tetid", "restlength", "restvector", "restdir")}

    def add(self, ctype, pts, k, damp, tetid, restlength, restvector=None, restdir=None):
        n = pts.shape[0]
        self.cols["type"].append(np.full(n, ctype, np.int32))
        self.cols["pts"].append(np.asarray(pts, np.int32).reshape(n, 4))
        self.cols["k"].append(np.full(n, k, np.float64) if np.isscalar(k) else np.asarray(k, np.float64))
        self.cols["damp"].append(np.full(n, damp, np.float64) if np.isscalar(damp) else np.asarray(damp, np.float64))
        self.cols["tetid"].append(np.asarray(tetid, np.int32))
        self.cols["restlength"].append(np.asarray(restlength, np.float64))
        self.cols["restvector"].append(np.zeros((n, 4)) if restvector is None else np.asarray(restvector, np.float64))
        self.cols["restdir"].append(np.zeros((n, 3)) if restdir is None else np.asarray(restdir, np.float64))

    @staticmethod
    def from_arrays(c_type, c_pts, c_stiffness, c_damp, c_tetid, c_restlength, c_restvector, c_restdir):
        """A table from reference struct-of-arrays columns (already in table order)."""
        t = Table()
        for k, v in zip(("type", "pts", "k", "damp", "tetid", "restlength", "restvector", "restdir"),
                        (c_type, c_pts, c_stiffness, c_damp, c_tetid, c_restlength, c_restvector, c_restdir)):
            t.cols[k].append(np.asarray(v))
        return t.finalize()

    def finalize(self):
        c = {k: (np.concatenate(v) if v else None) for k, v in self.cols.items()}
        if c["type"] is None:
            self.n = 0
            return self
        order = np.argsort(c["type"], kind="stable")
        for k in c:
            c[k] = c[k][order]
        self.c = c
        self.n = c["type"].shape[0]
        return self


def table_from_configs(pos0, tets, configs, tet_masks=None):
    """_collect_raw_constraints (builder.py:610-656) for the tet types."""
    V0, valid = signed_rest_volume(pos0, tets)
    t = Table()
    tet_masks = tet_masks or {}
    for prm in configs:
        if not prm.get("enable", True):
            continue
        ty = str(prm["type"]).lower()
        m = tet_masks.get(prm.get("name", ty))
        sel = valid if m is None else (valid & m)
        idx = np.nonzero(sel)[0]
        if "compliance" in prm:
            k = float("inf") if float(prm["compliance"]) == 0.0 else 1.0 / float(prm["compliance"])
        else:
            k = None
        d = float(prm.get("dampingratio", 0.0))
        if ty == "volume":
            t.add(T_TETVOLUME, tets[idx], k if k is not None else float(prm.get("stiffness", 1e10)), d, idx, V0[idx])
        elif ty in ("tetarapsvd", "aniso_arap"):
            t.add(T_TETARAPSVD if ty == "tetarapsvd" else T_TETARAPANISO, tets[idx],
                  k if k is not None else float(prm.get("stiffness", 1e6)), d, idx, V0[idx])
        elif ty == "snh":
            mu = float(prm.get("mu", prm.get("stiffness", 1000.0)))
            lam = float(prm.get("lam", 10000.0))
            rd = np.zeros((idx.shape[0], 3))
            rd[:, 0] = lam
            t.add(T_TETSNH, tets[idx], mu, d, idx, V0[idx], restdir=rd)
    return t


class OracleSolver:
    """The reference substep on the oracle: state + Jacobi projection of a table."""

    def __init__(self, pos0, tets, table: Table, mass, stopped, B, *, dt, gravity_vec, veldamping=0.0,
                 quasi_static=False, relaxation=1.0, v_fiber=None, activation=None, tendonmask=None,
                 contraction_ratio=0.0, fiber_stiffness_scale=1.0, prec="f32"):
        P = self.P = Prec(prec)
        self.nv = pos0.shape[0]
        self.nt = tets.shape[0]
        self.tets = np.ascontiguousarray(tets, np.int32)
        self.pos = P.arr(pos0, (self.nv, 3)).copy()
        self.pprev = self.pos.copy()
        self.vel = np.zeros_like(self.pos)
        self.mass = P.arr(mass)
        self.stopped = np.ascontiguousarray(stopped, np.int32)
        self.B = P.arr(B, (self.nt, 9))
        self.dt, self.g = float(dt), P.arr(gravity_vec)
        self.veldamping, self.qs, self.omega = float(veldamping), int(bool(quasi_static)), float(relaxation)
        self.v_fiber = P.arr(v_fiber if v_fiber is not None else np.zeros((self.nv, 3)))
        self.activation = P.arr(activation if activation is not None else np.zeros(self.nt))
        self.tendonmask = P.arr(tendonmask if tendonmask is not None else np.zeros(self.nt))
        self.ratio, self.kscale = float(contraction_ratio), float(fiber_stiffness_scale)
        self.table = table
        self.dP = np.zeros_like(self.pos)
        self.dPw = np.zeros(self.nv, P.dt)
        if table.n:
            c = table.c
            self.c_type = np.ascontiguousarray(c["type"], np.int32)
            self.c_pts = np.ascontiguousarray(c["pts"], np.int32)
            self.c_k = P.arr(c["k"])
            self.c_d = P.arr(c["damp"])
            self.c_tetid = np.ascontiguousarray(c["tetid"], np.int32)
            self.c_rl = P.arr(c["restlength"])
            self.c_rv = P.arr(c["restvector"], (table.n, 4))
            self.c_rd = P.arr(c["restdir"], (table.n, 3))
            L = lib()
            sz = getattr(L, f"orc_csr_size_{prec}")
            sz.restype = C.c_long
            nslot = sz(table.n, _p(self.c_type), _p(self.c_pts))
            self.row = np.zeros(self.nv + 1, np.int64)
            self.slot = np.zeros(nslot, np.int64)
            getattr(L, f"orc_build_csr_{prec}")(self.nv, table.n, _p(self.c_type), _p(self.c_pts), _p(self.row),
                                                 _p(self.slot))
            self.corr = np.zeros(12 * table.n, P.dt)
            self.cmask = np.zeros(table.n, np.int32)

    # reference primitives
    def integrate(self):
        f = self.P.fn("orc_integrate")
        f.argtypes = [C.c_int] + [C.c_void_p] * 7 + [self.P.ct, self.P.ct, C.c_int]
        f(self.nv, _p(self.pos), _p(self.pprev), _p(self.vel), None, _p(self.mass), _p(self.stopped), _p(self.g),
          self.P.ct(self.veldamping), self.P.ct(self.dt), self.qs)

    def update_velocities(self):
        if self.qs:
            return
        f = self.P.fn("orc_update_velocities")
        f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, self.P.ct]
        f(self.nv, _p(self.pos), _p(self.pprev), _p(self.vel), self.P.ct(self.dt))

    def project(self):
        """clear + solve_constraints (Jacobi): fills dP/dPw."""
        if not self.table.n:
            self.dP[:] = 0
            self.dPw[:] = 0
            return
        f = self.P.fn("orc_project")
        ct = self.P.ct
        f.argtypes = ([C.c_int] + [C.c_void_p] * 8 + [C.c_int] + [C.c_void_p] * 8 + [ct, ct, ct] + [C.c_void_p] * 6)
        f(self.nv, _p(self.pos), _p(self.pprev), _p(self.mass), _p(self.stopped), _p(self.B), _p(self.v_fiber),
          _p(self.activation), _p(self.tendonmask), self.table.n, _p(self.c_type), _p(self.c_pts), _p(self.c_k),
          _p(self.c_d), _p(self.c_tetid), _p(self.c_rl), _p(self.c_rv), _p(self.c_rd), ct(self.dt), ct(self.ratio),
          ct(self.kscale), _p(self.row), _p(self.slot), _p(self.corr), _p(self.cmask), _p(self.dP), _p(self.dPw))

    def apply_dP(self):
        f = self.P.fn("orc_apply_dP")
        f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, self.P.ct]
        f(self.nv, _p(self.pos), _p(self.dP), _p(self.dPw), self.P.ct(self.omega))

    def svd_clamp(self, sigma_min, alpha, iters):
        """XpbdEngine.repair_inverted_tets (engine.py:831-856): iters passes of
        _svd_clamp_accumulate_kernel (engine.py:293-367) and
        _apply_svd_clamp_kernel (engine.py:370-380).  The sign-fixed SVD (U, V
        rotations, s sorted descending, sign(s2) = sign(det F)) and the target
        edges are taken in float64; the per-vertex sums are added in tet order in
        the oracle's precision."""
        if alpha <= 0.0 or iters <= 0:
            return
        P = self.P
        t = self.tets.astype(np.int64)
        B = self.B.reshape(-1, 3, 3).astype(np.float64)
        Dm = np.linalg.inv(B)
        free = self.stopped == 0
        for _ in range(iters):
            x = self.pos
            c = np.stack([x[t[:, k]] - x[t[:, 3]] for k in range(3)], -1).astype(P.dt)  # columns p_k - p3
            F = np.einsum("nij,njk->nik", c.astype(np.float64), B)
            U, sv, Vt = np.linalg.svd(F)
            fu = np.linalg.det(U) < 0
            U[fu, :, 2] *= -1
            sv[fu, 2] *= -1
            fv = np.linalg.det(Vt) < 0
            Vt[fv, 2, :] *= -1
            sv[fv, 2] *= -1
            bad = (sv < sigma_min).any(1)
            dP = np.zeros_like(self.pos)
            w = np.zeros(self.nv, P.dt)
            if bad.any():
                Ft = np.einsum("nij,nj,njk->nik", U[bad], np.maximum(sv[bad], sigma_min), Vt[bad])
                Dt = np.einsum("nij,njk->nik", Ft, Dm[bad])
                d = Dt - c[bad].astype(np.float64)
                shift = (d[:, :, 0] + d[:, :, 1] + d[:, :, 2]) * 0.25
                corr = np.stack([d[:, :, 0] - shift, d[:, :, 1] - shift, d[:, :, 2] - shift, -shift], 1).astype(P.dt)
                tb = t[bad]
                for k in range(4):
                    m = free[tb[:, k]]
                    np.add.at(dP, tb[m, k], corr[m, k])
                    np.add.at(w, tb[m, k], P.dt(1))
            on = w > 0
            self.pos[on] = (self.pos[on] + (P.dt(alpha) * dP[on]) / w[on, None]).astype(P.dt)

    # metrics
    def count_inverted(self):
        f = self.P.fn("orc_count_inverted")
        return int(f(self.nt, _p(self.tets), _p(self.pos), _p(self.B)))

    def total_volume(self):
        f = self.P.fn("orc_total_volume")
        f.restype = C.c_double
        return float(f(self.nt, _p(self.tets), _p(self.pos)))

    def arap_residual(self):
        out = np.zeros(self.nt, self.P.dt)
        self.P.fn("orc_arap_residual")(self.nt, _p(self.tets), _p(self.pos), _p(self.B), _p(out))
        return out


class OracleMuscleSim(OracleSolver):
    """MuscleSim.from_procedural + step() (musclesim.py:107-142, 181-287) on the oracle."""

    def __init__(self, vertices, tets, fiber_dirs_per_tet, *, constraint_configs, dts, num_substeps=1,
                 density=1060.0, veldamping=0.02, gravity=0.0, stopped=None, relaxation=1.0,
                 contraction_ratio=0.0, fiber_stiffness_scale=1.0, tet_masks=None, repair_alpha=0.0, repair_iters=0,
                 repair_sigma_min=0.1, attach=None, prec="f32"):
        vertices = np.asarray(vertices, np.float32)
        tets = np.asarray(tets, np.int32)
        nv = vertices.shape[0]
        fd = np.asarray(fiber_dirs_per_tet, np.float32).reshape(-1, 3)
        vf = np.zeros((nv, 3), np.float32)
        vc = np.zeros(nv, np.float32)
        for e, t in enumerate(tets):  # musclesim.py:226-234, same accumulation order
            for vi in t:
                vf[vi] += fd[e]
                vc[vi] += 1.0
        vc = np.maximum(vc, 1.0)
        vf /= vc[:, None]
        vf /= np.maximum(np.linalg.norm(vf, axis=1, keepdims=True), 1e-8)
        rv, B, mass, tot = precompute_rest(vertices, tets, density, prec)
        self.total_rest_volume = tot
        table = table_from_configs(vertices, tets, constraint_configs, tet_masks)
        if attach is not None:
            # bone attach rows (builder.py:347-398): (src, target xyz, rest length, stiffness, damping)
            src, tgt, rl, k, d = attach
            n = len(src)
            pts = np.full((n, 4), -1, np.int32)
            pts[:, 0] = src
            rv = np.ones((n, 4))
            rv[:, :3] = tgt
            table.add(T_ATTACH, pts, float(k), float(d), np.full(n, -1), np.asarray(rl, np.float64), restvector=rv)
        table = table.finalize()
        st = np.zeros(nv, np.int32) if stopped is None else np.asarray(stopped, np.int32)
        super().__init__(vertices, tets, table, mass, st, B, dt=float(dts) / int(num_substeps),
                         gravity_vec=(0.0, float(gravity), 0.0), veldamping=veldamping, relaxation=relaxation,
                         v_fiber=vf, contraction_ratio=contraction_ratio,
                         fiber_stiffness_scale=fiber_stiffness_scale, prec=prec)
        self.num_substeps = int(num_substeps)
        self.repair = (float(repair_sigma_min), float(repair_alpha), int(repair_iters))

    def substep(self):
        """integrate_phase, solve_phase, finalize_phase (musclesim.py:107-130)
        with the SVD inversion repair before the velocity update."""
        self.integrate()
        self.project()
        self.apply_dP()
        self.svd_clamp(*self.repair)
        self.update_velocities()

    def step(self):
        for _ in range(self.num_substeps):
            self.substep()


def sdf_bake(nxyz, origin, h, caps, transforms, band, prec="f32"):
    """Capsule-union SDF on the grid, clamped to band (see orc_sdf_bake_capsules)."""
    P = Prec(prec)
    nx, ny, nz = nxyz
    phi = np.zeros((nz, ny, nx), P.dt)
    f = P.fn("orc_sdf_bake_capsules")
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, P.ct, C.c_int, C.c_void_p, C.c_void_p, P.ct, C.c_void_p]
    o = P.arr(origin)
    cp = P.arr(caps)
    tr = None if transforms is None else P.arr(transforms)
    f(nx, ny, nz, _p(o), P.ct(h), cp.shape[0], _p(cp), _p(tr), P.ct(band), _p(phi))
    return phi


def sdf_push(pos, inv_mass, phi, origin, h, offset, max_push, prec="f32"):
    P = Prec(prec)
    nz, ny, nx = phi.shape
    f = P.fn("orc_sdf_push")
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, P.ct, P.ct, P.ct]
    o = P.arr(origin)
    f(pos.shape[0], _p(pos), _p(P.arr(inv_mass)), _p(P.arr(phi)), nx, ny, nz, _p(o), P.ct(h), P.ct(offset),
      P.ct(max_push))


def _find(cfg, name):
    for c in cfg.get("constraints", []):
        if c.get("name") == name:
            return c if c.get("enable", True) else None
    return None


class OracleMultiGridSim(OracleSolver):
    """MultiGridSim's program (mg/mg.py:1322-1418) on the oracle, for a synthetic
    scene whose vertices ride capsule bones rigidly (rest_offset = 0)."""

    def __init__(self, cfg, scene, prec="f32", sdf_margin=0.02, band_cells=3.0):
        self.cfg, self.scene = cfg, scene
        verts, tets = scene.verts.astype(np.float32), scene.tets.astype(np.int32)
        nv, nt = verts.shape[0], tets.shape[0]
        arap = _find(cfg, "arap")
        snh = _find(cfg, "snh")
        fib = _find(cfg, "fiber")
        vol = _find(cfg, "volume")
        fascia = scene.tet_part < 0
        cons, masks = [], {}
        if snh:
            cons.append(dict(type="snh", name="snh", mu=float(snh.get("mu", snh.get("stiffness", arap["stiffness"]))),
                             lam=float(snh.get("lam", 1e8)), dampingratio=float(snh.get("dampingratio", 0.0))))
            if snh.get("region", "all") == "fascia":
                masks["snh"], masks["arap"] = fascia, ~fascia
                cons.append(dict(type="tetarapsvd", name="arap", stiffness=arap["stiffness"]))
        else:
            cons.append(dict(type="tetarapsvd", name="arap", stiffness=arap["stiffness"]))
        if vol and not (snh and snh.get("region", "all") == "all"):
            cons.append(dict(type="volume", name="volume", stiffness=vol["stiffness"],
                             dampingratio=vol.get("dampingratio", 0.0)))
            if snh:
                masks["volume"] = ~fascia
        if fib:
            cons.append(dict(type="aniso_arap", name="fiber", stiffness=float(fib.get("stiffness", 1e8))))
            if fib.get("region", "all") == "aniso_muscle":
                masks["fiber"] = scene.tet_part == scene.aniso_muscle
        self.contraction = float((fib or {}).get("contraction_ratio", 0.4))
        t = table_from_configs(verts, tets, cons, masks)
        V0, valid = signed_rest_volume(verts, tets)
        if cfg.get("density") is not None:
            rho = float(cfg["density"])
        else:
            rho = float(cfg["total_mass"]) / float(V0[valid].astype(np.float64).sum())
        rv, B, mass, tot = precompute_rest(verts, tets, rho, prec)
        self.total_rest_volume = tot
        pin = _find(cfg, "muscleToBonePin")
        self.active = np.zeros(nv, bool)
        if pin is not None and pin.get("region", "tendonmask") == "tendonmask":
            self.active = scene.v_tendon > float(pin["tendon_pin_threshold"])
        elif pin is not None and pin.get("region") == "full":
            self.active[:] = True
        belly = _find(cfg, "belly_attach")
        self.belly_src = np.nonzero(~self.active)[0] if belly else np.zeros(0, np.int64)
        if belly and self.belly_src.size:
            n = self.belly_src.shape[0]
            pts = np.full((n, 4), -1, np.int32)
            pts[:, 0] = self.belly_src
            t.add(T_ATTACH, pts, float(belly["stiffness"]), float(belly.get("dampingratio", 0.0)), np.full(n, -1),
                  np.zeros(n), restvector=np.ones((n, 4)))
        t.finalize()
        tendon_tet = (scene.v_tendon[tets].astype(np.float32).sum(1) / np.float32(4.0)).astype(np.float32)
        self.nsub = int(cfg["nsubsteps"])
        self.fine_iters = int(cfg["fine_iterations"])
        super().__init__(verts, tets, t, mass, np.zeros(nv, np.int32), B, dt=float(cfg["delta_t"]) / self.nsub,
                         gravity_vec=cfg.get("gravity", [0, 0, 0]), veldamping=float(cfg.get("veldamping", 0.0)),
                         quasi_static=bool(cfg.get("quasi_static", False)), v_fiber=scene.v_fiber,
                         tendonmask=tendon_tet, contraction_ratio=self.contraction, prec=prec)
        if t.n:
            self.attach_rows = np.nonzero(self.c_type == T_ATTACH)[0]
            order = np.argsort(self.c_pts[self.attach_rows, 0])
            self.attach_rows = self.attach_rows[order]
        coll = (cfg.get("demo") or {}).get("collision") or {}
        self.coll = coll if coll.get("enabled", False) else None
        if self.coll:
            lo, hi = verts.min(0) - sdf_margin, verts.max(0) + sdf_margin
            res = int(coll.get("sdf_res", 256))
            self.sdf_h = float((hi - lo).max()) / (res - 1)
            self.sdf_origin = lo.astype(np.float64)
            self.sdf_res = res
            self.band = band_cells * self.sdf_h
            self.caps = np.concatenate([scene.bone_center, scene.bone_half[:, None], scene.bone_axis,
                                        scene.bone_radius[:, None]], 1)
        self.inv_mass = np.where(self.mass > 0, 1.0 / np.where(self.mass > 0, self.mass, 1), 0).astype(self.P.dt)
        self.target = None
        self.mg = None
        scfg = (cfg.get("demo") or {}).get("self_collision") or {}
        self.dcd = scfg if str(scfg.get("method", "none")).lower() == "udcf" else None
        # soft pin of every vertex toward its target after the hard pin, once per
        # kinematic step (mg.py:133, 1386-1397; presubframe_pintotarget_kernel,
        # mg/kernel.py:229-257)
        self.presub = float(cfg.get("presubframe_pintotarget", 0.0))
        if cfg.get("use_multigrid", False):
            self._init_mg(float(arap["stiffness"]))

    # ---- multigrid (mg/mg.py:744-1079, mg/kernel.py:8-178) --------------------
    def _init_mg(self, mu):
        from rlmusclev2_b200.meshgen import cage_for_config  # input geometry only
        cfg, P = self.cfg, self.P
        cage = cage_for_config(self.scene, cfg, operator=str(cfg.get("mg_restrict_operator", "tikhonov")))
        # "residual": prior + Minv P^T (x - P prior); "direct": Minv P^T x, the
        # reference's scatter + block solve (mg/kernel.py:137-178) as written
        self.mg_form = str(cfg.get("mg_restrict_form", "residual"))
        self.cage = cage
        emb = np.nonzero(cage.cage_idx >= 0)[0]
        self.mg_emb = emb
        self.mg_t = cage.coarse_tet[cage.cage_idx[emb]]
        u = cage.uvw[emb].astype(P.dt)
        self.mg_w = np.concatenate([(P.dt(1) - u[:, 0] - u[:, 1] - u[:, 2])[:, None], u], 1)
        nc = cage.coarse_pos.shape[0]
        starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
        self.mg_blocks = [(int(cage.blk_base[s0]), int(cage.blk_dim[s0]),
                           cage.minv_flat[cage.blk_matoff[s0]:cage.blk_matoff[s0] + cage.blk_dim[s0] ** 2]
                           .astype(P.dt).reshape(cage.blk_dim[s0], cage.blk_dim[s0])) for s0 in starts]
        q0 = self.restrict(self.scene.verts.astype(P.dt), cage.coarse_pos.astype(P.dt)).astype(np.float32)
        self.mg_target = q0.astype(P.dt).copy()
        r = q0[cage.coarse_tet].astype(np.float64)  # _rest_B_p3ref (mg.py:43-53)
        Dm = np.stack([r[:, 0] - r[:, 3], r[:, 1] - r[:, 3], r[:, 2] - r[:, 3]], axis=-1)
        B = np.linalg.inv(Dm).astype(np.float32)
        rp = cage.coarse_pos[cage.coarse_tet].astype(np.float64)  # _node_mass_redistribute (mg.py:56-68)
        vol = np.abs(np.linalg.det(np.stack([rp[:, 1] - rp[:, 0], rp[:, 2] - rp[:, 0], rp[:, 3] - rp[:, 0]], -1))) / 6
        m = np.zeros(nc)
        np.add.at(m, cage.coarse_tet.reshape(-1), np.repeat(vol / 4.0, 4))
        m *= float(cfg["total_mass"]) / m.sum()
        w4 = np.abs(self.mg_w.astype(np.float64))
        wacc, pacc = np.zeros(nc), np.zeros(nc)
        np.add.at(wacc, self.mg_t.reshape(-1), w4.reshape(-1))
        np.add.at(pacc, self.mg_t.reshape(-1), (self.active[emb].astype(np.float64)[:, None] * w4).reshape(-1))
        with np.errstate(divide="ignore", invalid="ignore"):
            frac = np.where(wacc > 1e-9, pacc / wacc, 0.0)
        pin = ((frac >= float(cfg.get("mg_coarse_pin_frac", 0.5))) & (wacc > 1e-9)).astype(np.int32)
        self.mg_pin = pin.astype(bool)
        # coarse soft attach of the nodes with a nonzero restriction column after
        # every coarse sweep (mg.py:216, 836-841, 1047-1062)
        self.mg_beta = float(cfg.get("mg_coarse_attach_beta", 0.0))
        self.mg_attach = wacc > 1e-9
        t = Table()
        V0, _ = signed_rest_volume(q0, cage.coarse_tet)
        t.add(T_TETARAPSVD, cage.coarse_tet, mu, 0.0, np.arange(cage.coarse_tet.shape[0]), V0)
        t.finalize()
        self.mg = OracleSolver(q0, cage.coarse_tet, t, m.astype(np.float32), pin, B, dt=self.dt, gravity_vec=(0, 0, 0),
                               prec=P.name)
        self.mg_iters = int(cfg.get("mg_coarse_iters", 15))
        # step 1 of the V-cycle (mg.py:224-246, 1006-1012) and the coarse-in-fine
        # embedding of the "c2f" state restriction (mg.py:897-938)
        self.mg_restrict_mode = str(cfg.get("mg_restrict_mode", "direct")).lower()
        self.mg_sync = str(cfg.get("mg_sync_restrict", "galerkin")).lower()
        if self.mg_sync == "c2f":
            from rlmusclev2_b200.meshgen import coarse_in_fine_embedding  # input geometry only
            ct, cw = coarse_in_fine_embedding(self.scene.verts.astype(np.float32), self.scene.tets, cage.coarse_pos)
            self.mg_c2f = (ct.astype(np.int64), cw.astype(P.dt))

    def restrict(self, x, prior):
        """Regularised Galerkin restriction prior + Minv P^T (x - P prior)
        (restrict_galerkin_scatter_kernel + block_solve_kernel with the prior
        term; serial scatter in fine order)."""
        P = self.P
        nc = self.cage.coarse_pos.shape[0]
        prior = prior.astype(P.dt)
        if getattr(self, "mg_form", "residual") == "direct":
            prior = np.zeros_like(prior)
        w, t = self.mg_w, self.mg_t
        xe = x[self.mg_emb].astype(P.dt)
        r = xe - (((w[:, 0:1] * prior[t[:, 0]] + w[:, 1:2] * prior[t[:, 1]]) + w[:, 2:3] * prior[t[:, 2]])
                  + w[:, 3:4] * prior[t[:, 3]])
        b = np.zeros((nc, 3), P.dt)
        for k in range(4):
            np.add.at(b, t[:, k], w[:, k:k + 1] * r)
        out = np.zeros_like(b)
        for base, dim, M in self.mg_blocks:
            out[base:base + dim] = M @ b[base:base + dim]
        return prior + out

    def blend(self, pos, tgt, beta):
        """pos + beta (tgt - pos) with one rounding per component, as the device's
        fma (the FP32 product is exact in float64)."""
        P = self.P
        d = (tgt.astype(P.dt) - pos).astype(P.dt)
        return (pos.astype(np.float64) + np.float64(P.dt(beta)) * d.astype(np.float64)).astype(P.dt)

    def vcycle(self):
        """_hpbd_vcycle (mg.py:1064-1079): restrict, kinematic pin, coarse sweeps
        each followed by the soft attach when mg_coarse_attach_beta != 0
        (dense_soft_attach_kernel, mg/kernel.py:64-84), delta prolongation.
        With mg_mode "projection" (mg.py:1263-1320): the restricted bone target
        prolonged absolute onto the embedded fine vertices (prolong_kernel,
        mg/kernel.py:181-203)."""
        if str(self.cfg.get("mg_mode", "hpbd")).lower() == "projection":
            c, w, t, e = self.mg_target, self.mg_w, self.mg_t, self.mg_emb
            self.pos[e] = (((w[:, 0:1] * c[t[:, 0]] + w[:, 1:2] * c[t[:, 1]]) + w[:, 2:3] * c[t[:, 2]])
                           + w[:, 3:4] * c[t[:, 3]]).astype(self.P.dt)
            return
        co = self.mg
        if self.mg_restrict_mode == "direct" and self.mg_sync == "c2f":
            t, w = self.mg_c2f  # restrict_c2f_kernel (mg/kernel.py:43-60)
            x = self.pos
            co.pos[:] = (((w[:, 0:1] * x[t[:, 0]] + w[:, 1:2] * x[t[:, 1]]) + w[:, 2:3] * x[t[:, 2]])
                         + w[:, 3:4] * x[t[:, 3]]).astype(self.P.dt)
        elif self.mg_restrict_mode == "direct":
            co.pos[:] = self.restrict(self.pos, co.pos)
        elif self.mg_restrict_mode == "galerkin":  # the restricted bone target (mg.py:1265-1295)
            co.pos[:] = self.mg_target
        prev = co.pos.copy()
        tgt = self.mg_target
        co.pos[self.mg_pin] = tgt[self.mg_pin]
        for _ in range(self.mg_iters):
            co.project()
            co.apply_dP()
            if self.mg_beta != 0.0:
                m = self.mg_attach
                co.pos[m] = self.blend(co.pos[m], tgt[m], self.mg_beta)
        d = co.pos - prev
        e = self.mg_emb
        w = self.mg_w
        self.pos[e] += ((w[:, 0:1] * d[self.mg_t[:, 0]] + w[:, 1:2] * d[self.mg_t[:, 1]]) + w[:, 2:3] * d[self.mg_t[:, 2]]) \
            + w[:, 3:4] * d[self.mg_t[:, 3]]

    def targets(self, frame):
        """Two-bone blended target (1-w)(R_a x + t_a) + w (R_b x + t_b), float32."""
        T = self.scene.bone_transforms(frame).astype(np.float32)
        x = self.scene.verts.astype(np.float32)
        outs = []
        for k in range(2):
            Tb = T[self.scene.vert_bone[:, k]]
            o = np.empty_like(x)
            for r in range(3):
                o[:, r] = ((Tb[:, r, 0] * x[:, 0] + Tb[:, r, 1] * x[:, 1]) + Tb[:, r, 2] * x[:, 2]) + Tb[:, r, 3]
            outs.append(o)
        w = self.scene.vert_bw.astype(np.float32)[:, None]
        return (outs[0] + w * (outs[1] - outs[0])).astype(np.float32), T.reshape(-1, 12)

    def dcd_solve(self, it):
        """UdcfDcdCollider.solve (udcf/solver.py:365-440) on the muscle surface, FP32."""
        c = self.dcd
        p4 = np.zeros((self.nv, 4), np.float32)
        p4[:, :3] = self.pos
        p4[:, 3] = self.inv_mass
        tris = self.scene.surface_tris
        if it == 0:
            self.dcd_prev = p4.copy()
            self.dcd_pairs, _ = dcd_pairs(tris, p4, float(c.get("thickness", 0.0)), bool(c.get("allow_self", True)))
        ids, data = dcd_narrow(self.dcd_pairs, tris, p4, float(c.get("offset", 1e-6)))
        out = dcd_respond_apply(ids, data, p4, self.dcd_prev, float(c.get("multiplier", 1.01)),
                                float(c.get("friction_static", 0.5)), float(c.get("friction_dynamic", 0.4)),
                                float(c.get("max_push", 0.0)))
        self.pos[:] = out[:, :3]
        self.dcd_last = (self.dcd_pairs.shape[0], ids.shape[0])

    def apply_pins(self):
        self.pos[self.active] = self.target[self.active]

    def step_frame(self, frame):
        self.target, T = self.targets(frame)
        if self.table.n and self.attach_rows.size:
            self.c_rv[self.attach_rows, :3] = self.target[self.c_pts[self.attach_rows, 0]]
        if self.scene.tet_part is not None and hasattr(self.scene, "activation"):
            self.activation[:] = self.scene.activation(frame)
        if self.mg is not None:
            # coarse Dirichlet targets, restricted once per target change (mg.py:1028-1045)
            self.mg_target = self.restrict(self.target, self.mg_target)
        self.apply_pins()
        if self.presub > 0.0:
            self.pos[:] = self.blend(self.pos, self.target, self.presub)
        if self.coll:
            self._sdf_bake(T)
        for _ in range(self.nsub):
            self.integrate()
            if self.mg is not None:
                self.vcycle()
            self.apply_pins()
            for it in range(self.fine_iters):
                self.project()
                self.apply_dP()
                self.apply_pins()
                if self.dcd is not None:
                    self.dcd_solve(it)
            if self.coll:
                self._sdf_push()
            self.update_velocities()

    def _sdf_bake(self, T):
        r = self.sdf_res
        self.phi = sdf_bake((r, r, r), self.sdf_origin, self.sdf_h, self.caps, T, self.band, self.P.name)

    def _sdf_push(self):
        sdf_push(self.pos, self.inv_mass, self.phi, self.sdf_origin, self.sdf_h,
                 float(self.coll.get("contact_offset", 0.0)), float(self.coll.get("max_push", -1.0)), self.P.name)


class OracleBatchSim(OracleMultiGridSim):
    """The batched-instance program on the oracle: the same substep over a
    BatchScene, each instance pushed out of its own capsule grid."""

    def __init__(self, cfg, scene, prec="f32", band_cells=3.0):
        super().__init__(cfg, scene, prec=prec)
        if self.coll:
            self.sdf_res = int(scene.sdf_res)
            self.band = band_cells * float(scene.sdf_frame[:, 3].max())

    def _sdf_bake(self, T):
        sc, r = self.scene, self.sdf_res
        self.phis = []
        for i in range(sc.n_inst):
            fr = sc.sdf_frame[i].astype(np.float64)
            self.phis.append(sdf_bake((r, r, r), fr[:3], float(fr[3]), self.caps[2 * i:2 * i + 2],
                                      T[2 * i:2 * i + 2], self.band, self.P.name))

    def _sdf_push(self):
        sc = self.scene
        off, mp = float(self.coll.get("contact_offset", 0.0)), float(self.coll.get("max_push", -1.0))
        for i in range(sc.n_inst):
            v0, v1 = int(sc.inst_vptr[i]), int(sc.inst_vptr[i + 1])
            fr = sc.sdf_frame[i].astype(np.float64)
            sub = np.ascontiguousarray(self.pos[v0:v1])
            sdf_push(sub, np.ascontiguousarray(self.inv_mass[v0:v1]), self.phis[i], fr[:3], float(fr[3]), off, mp,
                     self.P.name)
            self.pos[v0:v1] = sub


# ---- DCD (collision/udcf/kernel.py) on the oracle, FP32 -------------------------
def dcd_pairs(tris, pos4, thickness=0.0, allow_self=True, group=None):
    L = lib()
    tris = np.ascontiguousarray(tris, np.int32)
    pos4 = np.ascontiguousarray(pos4, np.float32)
    n = tris.shape[0]
    boxes = np.zeros((n, 6), np.float32)
    L.orc_dcd_aabb.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]
    L.orc_dcd_aabb(n, _p(tris), _p(pos4), C.c_float(thickness), _p(boxes))
    cap = 1 << 16
    while True:
        pairs = np.zeros((cap, 2), np.int32)
        L.orc_dcd_pairs.restype = C.c_long
        L.orc_dcd_pairs.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_long]
        g = None if group is None else np.ascontiguousarray(group, np.int32)
        npairs = L.orc_dcd_pairs(n, _p(tris), _p(g), int(allow_self), _p(boxes), _p(pairs), cap)
        if npairs <= cap:
            return pairs[:npairs], boxes
        cap = int(npairs)


def dcd_narrow(pairs, tris, pos4, offset_eps=1e-6):
    L = lib()
    pairs = np.ascontiguousarray(pairs, np.int32)
    cap = max(1, pairs.shape[0])
    c_ids = np.zeros((cap, 8), np.int32)
    c_data = np.zeros((cap, 12), np.float32)
    L.orc_dcd_narrow.restype = C.c_long
    L.orc_dcd_narrow.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                 C.c_long]
    nc = L.orc_dcd_narrow(pairs.shape[0], _p(pairs), _p(np.ascontiguousarray(tris, np.int32)),
                          _p(np.ascontiguousarray(pos4, np.float32)), C.c_float(offset_eps), _p(c_ids), _p(c_data),
                          cap)
    return c_ids[:nc], c_data[:nc]


def dcd_respond_apply(c_ids, c_data, pos4, xprev4, multiplier=1.01, mu_s=0.5, mu_d=0.4, max_push=0.0, jacobi_avg=True):
    """Returns the new pos4 (input not modified)."""
    L = lib()
    out = np.ascontiguousarray(pos4, np.float32).copy()
    dP = np.zeros_like(out)
    L.orc_dcd_respond_apply.argtypes = [C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                        C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]
    L.orc_dcd_respond_apply(c_ids.shape[0], _p(np.ascontiguousarray(c_ids, np.int32)),
                            _p(np.ascontiguousarray(c_data, np.float32)), _p(out),
                            _p(np.ascontiguousarray(xprev4, np.float32)), out.shape[0], C.c_float(multiplier),
                            C.c_float(mu_s), C.c_float(mu_d), C.c_float(max_push), int(jacobi_avg), _p(dP))
    return out


# ------------------------------------------------ bone-surface binding (target_mode="mesh")
def _v4(a):
    a = np.asarray(a, np.float32)
    if a.shape[1] == 4:
        return np.ascontiguousarray(a)
    out = np.zeros((a.shape[0], 4), np.float32)
    out[:, :3] = a
    return out


def bone_bind(query, bone_verts, tris, max_dist):
    """bone_bind_kernel (mg/kernel.py:287-310), brute force: (face, uv, local4)."""
    L = lib()
    q4, b4 = _v4(query), _v4(bone_verts)
    tris = np.ascontiguousarray(tris, np.int32)
    n = q4.shape[0]
    face = np.zeros(n, np.int32)
    uv = np.zeros((n, 2), np.float32)
    loc = np.zeros((n, 4), np.float32)
    L.orc_bone_bind.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_float, C.c_void_p,
                                C.c_void_p, C.c_void_p]
    L.orc_bone_bind(n, _p(q4), _p(b4), tris.shape[0], _p(tris), C.c_float(max_dist), _p(face), _p(uv), _p(loc))
    return face, uv, loc


def bone_slide_targets(muscle, anchor_face, anchor_uv, bind_face, bind_uv, local4, slide_range, reproject, max_dist,
                       bone_verts, tris):
    """bone_slide_target_kernel (mg/kernel.py:313-347): returns (targets [n,3],
    bind_face, bind_uv, local4) with the binding updated by accepted slides."""
    L = lib()
    m4, b4 = _v4(muscle), _v4(bone_verts)
    tris = np.ascontiguousarray(tris, np.int32)
    bf = np.array(bind_face, np.int32)
    buv = np.array(bind_uv, np.float32)
    loc = np.array(local4, np.float32)
    n = m4.shape[0]
    tgt = np.zeros((n, 4), np.float32)
    L.orc_bone_slide_targets.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_float, C.c_int, C.c_float, C.c_void_p, C.c_int, C.c_void_p,
                                         C.c_void_p]
    L.orc_bone_slide_targets(n, _p(m4), _p(np.ascontiguousarray(anchor_face, np.int32)),
                             _p(np.ascontiguousarray(anchor_uv, np.float32)), _p(bf), _p(buv), _p(loc),
                             C.c_float(slide_range), int(reproject), C.c_float(max_dist), _p(b4), tris.shape[0],
                             _p(tris), _p(tgt))
    return tgt[:, :3], bf, buv, loc


def bone_pose(rest, vert_bone, transforms):
    """Rigid pose of bone-surface vertices: R_b x + t_b per vertex (float32)."""
    L = lib()
    r4 = _v4(rest)
    tr = np.ascontiguousarray(np.asarray(transforms, np.float32).reshape(-1, 12))
    out = np.zeros_like(r4)
    L.orc_bone_pose.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_bone_pose(r4.shape[0], _p(r4), _p(np.ascontiguousarray(vert_bone, np.int32)), _p(tr), _p(out))
    return out[:, :3]


def m2m_glue(pair_a, pair_b, restlen, compliance, pos4, dt, omega=1.0):
    """solve_m2m_glue_kernel (mg/kernel.py:350-394), sequential over the pairs."""
    L = lib()
    out = np.array(pos4, np.float32)
    L.orc_m2m_glue.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                               C.c_float]
    L.orc_m2m_glue(len(pair_a), _p(np.ascontiguousarray(pair_a, np.int32)), _p(np.ascontiguousarray(pair_b, np.int32)),
                   _p(np.ascontiguousarray(restlen, np.float32)), _p(np.ascontiguousarray(compliance, np.float32)),
                   _p(out), C.c_float(dt), C.c_float(omega))
    return out


def surface_bind(query, surf_verts, tris, max_dist):
    """fascia_bind_kernel (fascia/fascia.py:130-157): (face, uv, gap, ok)."""
    L = lib()
    q4, s4 = _v4(query), _v4(surf_verts)
    tris = np.ascontiguousarray(tris, np.int32)
    n = q4.shape[0]
    face, ok = np.zeros(n, np.int32), np.zeros(n, np.int32)
    uv, gap = np.zeros((n, 2), np.float32), np.zeros(n, np.float32)
    L.orc_surface_bind.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_float, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_surface_bind(n, _p(q4), _p(s4), tris.shape[0], _p(tris), C.c_float(max_dist), _p(face), _p(uv), _p(gap),
                       _p(ok))
    return face, uv, gap, ok


def surface_ride(bound, face, uv, gap, surf_verts, tris, fascia_pos):
    """fascia_ride_kernel (fascia/fascia.py:160-176) on a copy of fascia_pos."""
    L = lib()
    f4 = _v4(fascia_pos).copy()
    L.orc_surface_ride.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
    L.orc_surface_ride(len(bound), _p(np.ascontiguousarray(bound, np.int32)), _p(np.ascontiguousarray(face, np.int32)),
                       _p(np.ascontiguousarray(uv, np.float32)), _p(np.ascontiguousarray(gap, np.float32)),
                       _p(_v4(surf_verts)), _p(np.ascontiguousarray(tris, np.int32)), _p(f4))
    return f4[:, :3]


def fascia_advect(follow, target4, prev4, fascia4):
    """fascia_advect_bone_kernel (fascia/fascia.py:45-62): (fascia4, prev4) updated copies."""
    L = lib()
    f4, p4 = np.array(fascia4, np.float32), np.array(prev4, np.float32)
    L.orc_fascia_advect.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_fascia_advect(len(follow), _p(np.ascontiguousarray(follow, np.int32)),
                        _p(np.ascontiguousarray(target4, np.float32)), _p(p4), _p(f4))
    return f4, p4


def fascia_anchor(local, cons, offset4, target4, fascia4):
    """fascia_anchor_bone_kernel (fascia/fascia.py:65-80) on a copy."""
    L = lib()
    f4 = np.array(fascia4, np.float32)
    L.orc_fascia_anchor.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_fascia_anchor(len(local), _p(np.ascontiguousarray(local, np.int32)), _p(np.ascontiguousarray(cons, np.int32)),
                        _p(np.ascontiguousarray(offset4, np.float32)), _p(np.ascontiguousarray(target4, np.float32)),
                        _p(f4))
    return f4


def fascia_glue(pf, pm, restlen, compliance, fascia4, muscle4, dt, omega=1.0):
    """solve_glue_kernel (fascia/fascia.py:83-125), sequential, on a copy of muscle4."""
    L = lib()
    m4 = np.array(muscle4, np.float32)
    L.orc_fascia_glue.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_float, C.c_float]
    L.orc_fascia_glue(len(pf), _p(np.ascontiguousarray(pf, np.int32)), _p(np.ascontiguousarray(pm, np.int32)),
                      _p(np.ascontiguousarray(restlen, np.float32)), _p(np.ascontiguousarray(compliance, np.float32)),
                      _p(np.ascontiguousarray(fascia4, np.float32)), _p(m4), C.c_float(dt), C.c_float(omega))
    return m4


def set_arap_skip(v: float) -> None:
    """ARAP-SVD skip threshold on sum((sigma-1)^2) of both precisions: 0 the
    reference's 1e-12, > 0 that value, < 0 none (an exact rotation only).
    Process-wide state of the oracle library: restore 0 after use."""
    L = lib()
    for p in ("f32", "f64"):
        f = getattr(L, f"orc_set_arap_skip_{p}")
        f.argtypes = [C.c_double]
        f.restype = None
        f(float(v))
