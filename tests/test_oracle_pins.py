"""Pins the CPU oracle against the known answers the reference's own tests state.

The reference (chunleili/rlmuscleV2) cannot run here: its kernels need NVIDIA
Warp, and its frame goldens are Git-LFS pointers.  Its single-tet tests
(tests/test_lion_kernels.py:14-169) are restated for the current kernels,
which use pts[3] as the rest reference vertex (solve_kernels.py:1231) and the
Jacobi dP/dPw form (solve_kernels.py:52-56); the DCD response tests
(tests/test_udcf_dcd.py:191-236, 335-400) are in test_dcd.py.
"""
import numpy as np

from oracle import oracle as O

T_ARAP = O.T_TETARAPSVD


def _single_tet(rest, deformed, k=1.0e9, dt=0.004166, prec="f64"):
    tets = np.array([[0, 1, 2, 3]], np.int32)
    rv, B, mass, tot = O.precompute_rest(rest, tets, 1.0, prec)
    t = O.Table()
    V0, _ = O.signed_rest_volume(rest, tets)
    t.add(T_ARAP, tets, k, 0.0, np.array([0]), V0)
    t.finalize()
    s = O.OracleSolver(np.asarray(deformed), tets, t, np.ones(4), np.zeros(4, np.int32), B, dt=dt,
                       gravity_vec=(0, 0, 0), prec=prec)
    s.project()
    return s, B


# regular tet ordered so that pts[3] is the origin: Dm = I
REG = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]], np.float64)


def test_precompute_regular_tet():
    """test_lion_kernels.py:14-35: regular tet -> B = I, V0 = 1/6."""
    tets = np.array([[0, 1, 2, 3]], np.int32)
    for prec in ("f32", "f64"):
        rv, B, mass, tot = O.precompute_rest(REG, tets, 1.0, prec)
        np.testing.assert_allclose(B[0], np.eye(3), atol=1e-6)
        np.testing.assert_allclose(rv[0], 1.0 / 6.0, atol=1e-7)
        np.testing.assert_allclose(mass, np.full(4, 1.0 / 24.0), rtol=1e-6)
    V0, valid = O.signed_rest_volume(REG, tets)
    assert valid[0] and abs(V0[0] - 1.0 / 6.0) < 1e-7


def test_arap_identity_no_displacement():
    """test_lion_kernels.py:38-63: F = I -> constraint below threshold -> no correction."""
    s, _ = _single_tet(REG, REG)
    assert np.all(s.dP == 0) and np.all(s.dPw == 0)


def test_arap_uniform_stretch_contracts_edges():
    """test_lion_kernels.py:66-103: x1.1 stretch -> one iteration shrinks the edges."""
    s, _ = _single_tet(REG, REG * 1.1)
    assert np.all(s.dPw == 1)
    s.apply_dP()
    new = s.pos
    for a, b in ((0, 3), (1, 3), (2, 3), (0, 1)):
        assert np.linalg.norm(new[a] - new[b]) < np.linalg.norm(1.1 * (REG[a] - REG[b]))


def test_arap_asymmetric_tet_matches_numpy_reference():
    """test_lion_kernels.py:106-169, restated for the pt3 reference vertex and
    the Jacobi dP form: numpy sign-fixed SVD gradient vs the oracle."""
    rest = np.array([[2, 0.1, 0.2], [0.3, 1.5, -0.1], [-0.2, 0.4, 1.3], [0, 0, 0]], np.float64)
    deformed = rest.copy()
    deformed[0] += np.array([0.05, -0.03, 0.07])
    k, dt = 1.0e9, 0.004166
    s, B = _single_tet(rest, deformed, k=k, dt=dt)
    B = B[0]
    Ds = np.stack([deformed[0] - deformed[3], deformed[1] - deformed[3], deformed[2] - deformed[3]], 1)
    F = Ds @ B
    U, S, Vt = np.linalg.svd(F)
    if np.linalg.det(U) < 0:
        U[:, 2] *= -1
        S[2] *= -1
    V = Vt.T
    if np.linalg.det(V) < 0:
        V[:, 2] *= -1
        S[2] *= -1
    C = float(np.sqrt(((S - 1) ** 2).sum()))
    dCdF = U @ np.diag((S - 1) / C) @ V.T
    g = [dCdF @ B[0], dCdF @ B[1], dCdF @ B[2]]
    g.append(-(g[0] + g[1] + g[2]))
    g = np.stack(g)
    at = (1.0 / k) / (dt * dt)
    dL = -C / ((g * g).sum() + at)
    np.testing.assert_allclose(s.dP, dL * g, atol=1e-12, rtol=1e-9)
    np.testing.assert_array_equal(s.dPw, np.ones(4))


def test_svd_sign_convention_random():
    """ssvd_fn (solve_kernels.py:85-112): U, V rotations, |s| sorted, sign(s2) = sign(det F)."""
    rng = np.random.default_rng(7)
    for _ in range(300):
        F = rng.normal(size=(3, 3))
        if rng.random() < 0.3:
            F[:, 2] = F[:, 0] * rng.normal() + 1e-9 * rng.normal(size=3)  # near rank-2
        U, s, V = O.svd3(F, "f64")
        np.testing.assert_allclose(U @ np.diag(s) @ V.T, F, atol=1e-10)
        assert abs(np.linalg.det(U) - 1) < 1e-10 and abs(np.linalg.det(V) - 1) < 1e-10
        assert s[0] >= s[1] >= abs(s[2]) - 1e-12
        assert s[1] >= 0
        if abs(np.linalg.det(F)) > 1e-9:
            assert np.sign(s[2]) == np.sign(np.linalg.det(F))


def test_oracle_f32_matches_f64_one_frame():
    """The FP32 restatement stays within the parity tolerance of FP64 after 10 substeps."""
    from tests._cases import CFG1, CFG1_CONSTRAINTS, bbox_diag, cfg1_mesh
    m = cfg1_mesh()
    sims = [O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                              stopped=m.stopped, prec=p, **CFG1) for p in ("f32", "f64")]
    for s in sims:
        s.step()
    err = np.abs(sims[0].pos - sims[1].pos).max()
    assert err < 1e-5 * bbox_diag(m.verts) * 0.1, err


def test_oracle_deterministic_and_thread_independent():
    import os
    from tests._cases import CFG1, CFG1_CONSTRAINTS, cfg1_mesh
    m = cfg1_mesh()
    runs = []
    for _ in range(2):
        s = O.OracleMuscleSim(m.verts, m.tets, m.fiber_per_tet, constraint_configs=CFG1_CONSTRAINTS,
                              stopped=m.stopped, prec="f32", **CFG1)
        s.step()
        runs.append(s.pos.copy())
    np.testing.assert_array_equal(runs[0], runs[1])
