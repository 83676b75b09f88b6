"""Shared test cases (seeded synthetic inputs)."""
import numpy as np

from rlmusclev2_b200.meshgen import box_muscle

CFG1_CONSTRAINTS = [{"type": "tetarapsvd", "name": "arap", "compliance": 1e-7},
                    {"type": "volume", "name": "volume", "compliance": 0.0}]
CFG1 = dict(dts=1.0 / 24.0, num_substeps=10, density=1060.0, veldamping=0.02, gravity=-9.8)


def cfg1_mesh(**kw):
    return box_muscle(**kw)


def random_tet_mesh(n_cube=3, spacing=0.01, jitter=0.0015, seed=1):
    """Small jittered cube lattice (6 tets per hex) for kernel-level parity."""
    m = box_muscle(nx=n_cube, ny=n_cube, nz=n_cube, spacing=spacing, jitter=jitter, seed=seed, pin_frac=0.0)
    return m.verts, m.tets


def bbox_diag(x):
    return float(np.linalg.norm(x.max(0) - x.min(0)))
