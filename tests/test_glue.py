"""Muscle-to-muscle glue on the CPU: the pair builder's rules
(mg/mg.py:581-660) and the oracle's glue step (mg/kernel.py:350-394)."""
import numpy as np

from oracle import oracle as O
from rlmusclev2_b200.glue import build_m2m_pairs


def _two_blocks(gap=0.0015, n=6, h=0.002):
    g = np.stack(np.meshgrid(*[np.arange(n) * h] * 3, indexing="ij"), -1).reshape(-1, 3)
    b = g + np.array([n * h - h + gap, 0.0, 0.0])
    pos = np.concatenate([g, b]).astype(np.float32)
    vm = np.r_[np.zeros(len(g), int), np.ones(len(b), int)]
    return pos, vm


def test_pairs_cross_muscles_within_radius_once():
    pos, vm = _two_blocks()
    mask = np.ones(len(pos), np.float32)
    a, b, rest = build_m2m_pairs(pos, vm, mask, 0.5, 0.002, 8)
    assert a.size > 0
    assert (a < b).all() and (vm[a] != vm[b]).all()
    assert (rest <= 0.002 + 1e-7).all()
    np.testing.assert_allclose(rest, np.linalg.norm(pos[a] - pos[b], axis=1), rtol=1e-6)
    assert len(set(zip(a.tolist(), b.tolist()))) == a.size
    # masked-out vertices take no part; a zero mask gives no pairs
    m2 = mask.copy()
    m2[vm == 1] = 0.0
    assert build_m2m_pairs(pos, vm, m2, 0.5, 0.002, 8)[0].size == 0
    # a radius below the gap finds nothing
    assert build_m2m_pairs(pos, vm, mask, 0.5, 0.001, 8)[0].size == 0


def test_oracle_glue_step_moves_pairs_to_rest_length():
    rng = np.random.default_rng(2)
    n = 40
    p4 = np.zeros((2 * n, 4), np.float32)
    p4[:, :3] = rng.random((2 * n, 3))
    p4[:, 3] = 1.0
    p4[n:, 3] = np.where(rng.random(n) < 0.3, 0.0, 1.0)  # some stopped endpoints
    a, b = np.arange(n), np.arange(n, 2 * n)
    rest = (np.linalg.norm(p4[a, :3] - p4[b, :3], axis=1) * 0.8).astype(np.float32)
    out = O.m2m_glue(a, b, rest, np.zeros(n, np.float32), p4, 1.0 / 240.0, 1.0)
    # zero compliance, omega 1, disjoint pairs: every pair lands on its rest length
    np.testing.assert_allclose(np.linalg.norm(out[a, :3] - out[b, :3], axis=1), rest, rtol=1e-5)
    assert np.array_equal(out[n:][p4[n:, 3] == 0], p4[n:][p4[n:, 3] == 0])  # stopped ends stay put
