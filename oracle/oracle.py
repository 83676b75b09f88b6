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
                 contraction_ratio=0.0, fiber_stiffness_scale=1.0, tet_masks=None, prec="f32"):
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
        table = table_from_configs(vertices, tets, constraint_configs, tet_masks).finalize()
        st = np.zeros(nv, np.int32) if stopped is None else np.asarray(stopped, np.int32)
        super().__init__(vertices, tets, table, mass, st, B, dt=float(dts) / int(num_substeps),
                         gravity_vec=(0.0, float(gravity), 0.0), veldamping=veldamping, relaxation=relaxation,
                         v_fiber=vf, contraction_ratio=contraction_ratio,
                         fiber_stiffness_scale=fiber_stiffness_scale, prec=prec)
        self.num_substeps = int(num_substeps)

    def substep(self):
        self.integrate()
        self.project()
        self.apply_dP()
        self.update_velocities()

    def step(self):
        for _ in range(self.num_substeps):
            self.substep()
