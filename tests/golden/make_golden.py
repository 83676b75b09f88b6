"""Generates the golden fixtures in this folder from the reference's own
pure-numpy code (chunleili/rlmuscleV2, src/muscle/constraint/builder.py,
src/muscle/util/mesh_utils.py, src/muscle/util/activation.py,
src/muscle/defs.py).  Those modules need only numpy and scipy, so they are
imported from a checkout of the reference; the Warp kernels are not.

    python tests/golden/make_golden.py <reference checkout>

writes builder_small.npz.  The fixture is committed; the tests read only the
.npz and never the reference.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

CONFIGS = [
    {"type": "tetarapsvd", "name": "arap", "stiffness": 1.0e6, "dampingratio": 0.1},
    {"type": "volume", "name": "volume", "stiffness": 1.0e10, "dampingratio": 0.05},
    {"type": "aniso_arap", "name": "fiber", "stiffness": 1.0e8},
    {"type": "snh", "name": "snh", "mu": 2.0e4, "lam": 1.0e6, "dampingratio": 0.1},
]
FIELDS = ("type", "pts", "stiffness", "compressionstiffness", "dampingratio", "tetid", "L", "restlength",
          "restvector", "restdir")
DTYPES = dict(type=np.int32, pts=np.int32, stiffness=np.float32, compressionstiffness=np.float32,
              dampingratio=np.float32, tetid=np.int32, L=np.float32, restlength=np.float32, restvector=np.float32,
              restdir=np.float32)


def small_mesh(seed: int = 7):
    """3x2x2 hex lattice (spacing 5 mm, jitter U(-0.5,0.5) mm), 6 tets per hex,
    every other tet with pts[0]/pts[1] swapped (both windings), plus two
    degenerate tets: one with a repeated vertex, whose determinant rounds to
    a tiny non-zero value (the builder keeps it), and one with all four
    vertices equal (det = 0: the builder skips it)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz, h = 3, 2, 2, 0.005
    g = np.stack(np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij"), -1)
    pos = (g.reshape(-1, 3) * h + rng.uniform(-5e-4, 5e-4, (g.size // 3, 3))).astype(np.float32)
    vid = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    tets = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                c = [vid(i + a, j + b, k + d) for a in (0, 1) for b in (0, 1) for d in (0, 1)]
                # Kuhn split of the cube along the 0-7 diagonal
                for p in ((1, 3), (3, 2), (2, 6), (6, 4), (4, 5), (5, 1)):
                    tets.append([c[0], c[p[0]], c[p[1]], c[7]])
    tets = np.asarray(tets, np.int32)
    tets[::2, [0, 1]] = tets[::2, [1, 0]]
    tets = np.concatenate([tets, [[0, 0, 1, 2], [3, 3, 3, 3]]]).astype(np.int32)
    fib = rng.normal(size=pos.shape)
    fib /= np.linalg.norm(fib, axis=1, keepdims=True)
    return pos, tets, fib.astype(np.float32)


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from muscle.constraint.builder import ConstraintBuilderMixin
    from muscle.defs import ConstraintType
    from muscle.util.activation import RampActivationSource
    from muscle.util.mesh_utils import fix_tet_winding

    pos, tets, fib = small_mesh()

    class Host(ConstraintBuilderMixin):
        def __init__(self):
            self.pos0_np, self.tet_np, self.v_fiber_np = pos, tets, fib
            self.constraint_configs = CONFIGS

    host = Host()
    B, V, valid = host._batch_compute_tet_rest_matrices()
    cons, _ = host._collect_raw_constraints()
    cols = {f"c_{f}": np.array([c[f] for c in cons], dtype=DTYPES[f]) for f in FIELDS}
    mask = (np.arange(tets.shape[0]) % 3 == 0).astype(np.float32)
    ramp = RampActivationSource(mask, 1, 50)
    frames = np.arange(-2, 60, dtype=np.int32)
    acts = np.stack([ramp.per_tet(int(f)) for f in frames])
    np.savez_compressed(
        HERE / "builder_small.npz", pos0=pos, tets=tets, v_fiber=fib, rest_B=B, rest_V=V, rest_valid=valid,
        tets_fixed=fix_tet_winding(pos, tets[:-2]), act_mask=mask, act_frames=frames, act_values=acts,
        configs=np.array(json.dumps(CONFIGS)),
        ctype_names=np.array([m.name for m in ConstraintType]),
        ctype_values=np.array([int(m.value) for m in ConstraintType], np.int64), **cols)
    print(f"wrote {HERE / 'builder_small.npz'}: {tets.shape[0]} tets, {len(cons)} constraints")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
