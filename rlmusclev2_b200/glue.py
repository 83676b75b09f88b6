"""Muscle-to-muscle glue springs (MultiGridSim._build_m2m_glue, mg/mg.py:581-660):
rest-state pairs between adjacent muscles, solved on the device by
xpbd_m2m_glue (solve_m2m_glue_kernel, mg/kernel.py:350-394)."""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree


def build_m2m_pairs(pos0: np.ndarray, vert_muscle: np.ndarray, mask: np.ndarray, threshold: float = 0.5,
                    radius: float = 0.01, knn: int = 8):
    """Pairs (a, b), a < b, of glue-enabled vertices (mask > threshold) on
    different muscles, each vertex scanning its knn nearest enabled neighbours
    in rest-distance order: the first neighbour of another muscle within
    ``radius`` makes its pair, unless that pair exists already (then the scan
    ends without one); one pair per scanning vertex.  Returns (a, b, restlen)."""
    pos0 = np.asarray(pos0, np.float32)
    cand = np.nonzero(np.asarray(mask, np.float32) > threshold)[0].astype(np.int64)
    if cand.shape[0] < 2:
        return np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)
    cpos = pos0[cand]
    cm = np.asarray(vert_muscle)[cand]
    k = min(int(knn) + 1, cand.shape[0])
    dist, nbr = cKDTree(cpos).query(cpos, k=k)
    dist, nbr = np.atleast_2d(dist), np.atleast_2d(nbr)
    made: set[tuple[int, int]] = set()
    a_out, b_out = [], []
    for i in range(cand.shape[0]):
        for j, d in zip(nbr[i, 1:], dist[i, 1:]):
            if d > radius:
                break
            if cm[i] == cm[j]:
                continue
            key = tuple(sorted((int(cand[i]), int(cand[j]))))
            if key not in made:
                made.add(key)
                a_out.append(key[0])
                b_out.append(key[1])
            break
    a = np.asarray(a_out, np.int32)
    b = np.asarray(b_out, np.int32)
    restlen = np.linalg.norm(pos0[a] - pos0[b], axis=1).astype(np.float32) if a.size else np.zeros(0, np.float32)
    return a, b, restlen
