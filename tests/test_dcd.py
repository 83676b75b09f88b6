"""DCD oracle pinned to the reference's known answers (tests/test_udcf_dcd.py of
chunleili/rlmuscleV2: :191-236 response splits, :239-279 pair rules,
:282-332 penetration resolution, :335-400 friction slip)."""
import numpy as np

from oracle import oracle as O


def _contact(n, C, b1, b2, cur=(0, 1, 2), clo=(3, 4, 5)):
    ids = np.array([[*cur, 0, *clo, 0]], np.int32)
    data = np.zeros((1, 12), np.float32)
    data[0, :3], data[0, 3] = n, C
    data[0, 4:7], data[0, 8:11] = b1, b2
    return ids, data


X = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1], [0, 0.005, 0], [1, 0.005, 0], [0, 0.005, 1]], np.float32)
B3 = np.full(3, 1 / 3, np.float32)


def _pos4(x, im):
    p = np.zeros((x.shape[0], 4), np.float32)
    p[:, :3], p[:, 3] = x, im
    return p


def test_respond_solid_side_full_push():
    ids, data = _contact((0, 1, 0), 0.01, B3, B3)
    p = _pos4(X, [1, 1, 1, 0, 0, 0])
    out = O.dcd_respond_apply(ids, data, p, p, multiplier=1.01, mu_s=0.5, mu_d=0.4)
    assert np.allclose(out[0:3, 1], 0.01 * 1.01, atol=1e-6)
    assert np.allclose(out[3:6, :3], X[3:6], atol=1e-7)


def test_respond_both_movable_half_split():
    ids, data = _contact((0, 1, 0), 0.01, B3, B3)
    p = _pos4(X, np.ones(6))
    out = O.dcd_respond_apply(ids, data, p, p)
    half = 0.01 * 1.01 * 0.5
    assert np.allclose(out[0:3, 1] - X[0:3, 1], +half, atol=1e-6)
    assert np.allclose(out[3:6, 1] - X[3:6, 1], -half, atol=1e-6)


def test_respond_solid_side_friction_slipping():
    """Exact numbers of the reference's derivation: movable delta (-0.002, C*mult, 0)."""
    ids, data = _contact((0, 1, 0), 0.01, B3, B3)
    p = _pos4(X, [1, 1, 1, 0, 0, 0])
    prev = p.copy()
    prev[0:3, 0] -= 0.02
    out = O.dcd_respond_apply(ids, data, p, prev, multiplier=1.01, mu_s=0.5, mu_d=0.4)
    np.testing.assert_allclose(out[0:3, :3] - X[0:3], np.tile([-0.002, 0.0101, 0.0], (3, 1)), atol=1e-6)
    np.testing.assert_allclose(out[3:6, :3], X[3:6], atol=1e-7)


def test_pair_group_rules():
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1], [0.1, 0.01, 0.1], [1, 0.01, 1], [0, 0.02, 0], [1, 0.02, 0],
                  [0, 0.02, 1], [0, 0.03, 0], [1, 0.03, 0], [0, 0.03, 1]], np.float32)
    tris = np.array([[0, 1, 2], [1, 3, 4], [5, 6, 7], [8, 9, 10]], np.int32)
    group = np.array([0, 0, 1, 1], np.int32)
    p = _pos4(x, 1)
    for allow in (False, True):
        pairs, _ = O.dcd_pairs(tris, p, thickness=0.05, allow_self=allow, group=group)
        assert set(map(tuple, pairs.tolist())) == {(0, 2), (0, 3), (1, 2), (1, 3)}


def penetration_scene():
    mov = np.array([[-0.5, -0.02, -0.3], [0.5, 0.04, -0.3], [0.0, -0.02, 0.6]], np.float32)
    sta = np.array([[-1, 0, -1], [1, 0, -1], [0, 0, 1.5]], np.float32)
    x = np.concatenate([mov, sta])
    p = _pos4(x, [1, 1, 1, 0, 0, 0])
    tris = np.array([[0, 1, 2], [3, 4, 5]], np.int32)
    group = np.array([0, 1], np.int32)
    return p, tris, group


def test_collider_resolves_penetration():
    """A movable triangle tilted through a static one separates within 8 passes."""
    p, tris, group = penetration_scene()
    depth0 = -float(p[0:3, 1].min())
    pairs, _ = O.dcd_pairs(tris, p, 0.0, False, group)
    prev = p.copy()
    for it in range(8):
        ids, data = O.dcd_narrow(pairs, tris, p)
        p = O.dcd_respond_apply(ids, data, p, prev)
    assert pairs.shape[0] == 1
    assert -float(p[0:3, 1].min()) < depth0 * 0.5
