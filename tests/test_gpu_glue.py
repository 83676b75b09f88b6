"""Muscle-to-muscle glue on the GPU: xpbd_m2m_glue against the oracle's step
on pairs with distinct vertices (where the atomic and the sequential forms
agree), and MultiGridSim with a muscleToMuscleGlue block, which runs its fine
iterations in the reference's order (solve, average, glue, re-pin)."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from rlmusclev2_b200 import _capi as capi

pytestmark = pytest.mark.gpu


def test_glue_kernel_matches_oracle():
    lib = capi.load()
    rng = np.random.default_rng(5)
    n = 3000
    p4 = np.zeros((2 * n, 4), np.float32)
    p4[:, :3] = rng.random((2 * n, 3))
    p4[:, 3] = rng.uniform(0.5, 2.0, 2 * n)
    p4[rng.random(2 * n) < 0.1, 3] = 0.0
    perm = rng.permutation(2 * n)
    a, b = perm[:n].astype(np.int32), perm[n:].astype(np.int32)
    rest = (np.linalg.norm(p4[a, :3] - p4[b, :3], axis=1) * rng.uniform(0.5, 1.5, n)).astype(np.float32)
    comp = rng.uniform(0.0, 1e-6, n).astype(np.float32)
    dt, omega = 1.0 / 240.0, 0.7
    d = {k: torch.from_numpy(v).cuda() for k, v in dict(a=a, b=b, r=rest, c=comp, p=p4.copy()).items()}
    ptr = {k: C.c_void_p(v.data_ptr()) for k, v in d.items()}
    for _ in range(2):  # two calls in a row: the second starts from the first's result
        assert lib.xpbd_m2m_glue(n, ptr["a"], ptr["b"], ptr["r"], ptr["c"], ptr["p"], C.c_float(dt),
                                 C.c_float(omega), None) == 0
    torch.cuda.synchronize()
    ref = O.m2m_glue(a, b, rest, comp, O.m2m_glue(a, b, rest, comp, p4, dt, omega), dt, omega)
    got = d["p"].cpu().numpy()
    err = np.abs(got - ref).max()
    print(f"glue: |gpu - oracle| {err:.2e}")
    assert err < 1e-6
    assert np.array_equal(got[:, 3], p4[:, 3])


def test_multigrid_with_glue_steps():
    from rlmusclev2_b200.mg import MultiGridSim, load_config
    from rlmusclev2_b200.meshgen import humanv2_scene
    cfg = load_config("rlmusclev2_b200/configs/humanv2_synth.json")
    cfg["demo"]["collision"]["sdf_res"] = 96
    cfg["constraints"].append({"type": "muscleToMuscleGlue", "name": "muscleToMuscleGlue", "enable": True,
                               "region": "interface", "distance": 0.02, "stiffness": 1.0e6})
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    sim = MultiGridSim(cfg, scene=sc)
    assert sim.n_m2m > 0
    a, b = sim.m2m_pairs_user
    for frame in range(1, 4):
        sim.set_fiber_activation(sc.activation(frame))
        sim.step_frame(frame)
    p = sim.positions_np()
    assert np.isfinite(p).all()
    gap = np.linalg.norm(p[a] - p[b], axis=1)
    rest = np.linalg.norm(sim.pos0_np[a] - sim.pos0_np[b], axis=1)
    print(f"glue pairs {sim.n_m2m}: |gap - rest| max {np.abs(gap - rest).max():.2e} m")
    assert np.abs(gap - rest).max() < 0.02
