"""The coarse-cage baker (meshgen.build_cage), the project's stand-in for
tools/gen_coarse_cage.py: the same arrays with the same meaning
(mg/mg.py:770-800 reads them), and a valid embedding.

Checked on the config-3 scene (40 muscles, 16 mm lattice): every muscle
vertex is embedded and fascia vertices are not; barycentric weights sum to
one and are non-negative (each fine vertex lies inside its cage tet) and
reproduce the rest positions from the cage corners; every cage corner carries
fine weight (no unreferenced corner); each Galerkin block is symmetric
positive definite and the regularised operator restricts a state the cage can
represent back to itself.
"""
import numpy as np
import pytest

from rlmusclev2_b200.meshgen import build_cage
from rlmusclev2_b200.mg import load_config, scene_from_cfg

CFG3 = "rlmusclev2_b200/configs/humanv2_synth_mg_dcd.json"


@pytest.fixture(scope="module")
def scene_and_cage():
    cfg = load_config(CFG3)
    sc = scene_from_cfg(cfg)
    return sc, build_cage(sc, spacing=float(cfg.get("mg_cage_spacing", 0.016)))


def _weights(cage):
    emb = np.nonzero(cage.cage_idx >= 0)[0]
    u = cage.uvw[emb].astype(np.float64)
    w = np.concatenate([(1.0 - u.sum(1))[:, None], u], 1)
    return emb, cage.coarse_tet[cage.cage_idx[emb]], w


def test_arrays_follow_the_baked_cage_layout(scene_and_cage):
    sc, cage = scene_and_cage
    nv, nc = sc.verts.shape[0], cage.coarse_pos.shape[0]
    assert cage.cage_idx.dtype == np.int32 and cage.cage_idx.shape == (nv,)
    assert cage.uvw.dtype == np.float32 and cage.uvw.shape == (nv, 3)
    assert cage.coarse_pos.dtype == np.float32 and cage.coarse_tet.dtype == np.int32
    for a in (cage.blk_base, cage.blk_dim, cage.blk_matoff):
        assert a.dtype == np.int32 and a.shape == (nc,)
    assert cage.minv_flat.dtype == np.float32
    starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
    assert int((cage.blk_dim[starts].astype(np.int64) ** 2).sum()) == cage.minv_flat.shape[0]
    # blocks tile the coarse vertices in order
    assert np.array_equal(cage.blk_base[starts], np.r_[0, np.cumsum(cage.blk_dim[starts])[:-1]])


def test_embedding_is_valid(scene_and_cage):
    sc, cage = scene_and_cage
    muscle = sc.vert_part >= 0
    assert (cage.cage_idx[muscle] >= 0).all()
    assert (cage.cage_idx[~muscle] == -1).all()
    emb, t, w = _weights(cage)
    assert np.abs(w.sum(1) - 1.0).max() < 1e-6
    assert w.min() > -1e-5  # inside the cage tet up to FP32 rounding of uvw
    rec = (w[:, :, None] * cage.coarse_pos[t].astype(np.float64)).sum(1)
    assert np.abs(rec - sc.verts[emb]).max() < 2e-6
    # each cage tet embeds a fine vertex, so every corner carries weight
    nc = cage.coarse_pos.shape[0]
    wsum = np.zeros(nc)
    np.add.at(wsum, t.reshape(-1), np.abs(w).reshape(-1))
    assert (wsum > 0).all()
    # the cage tets of one muscle use only that muscle's block
    starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
    blk_of = np.searchsorted(cage.blk_base[starts], np.arange(nc), side="right") - 1
    assert (blk_of[t] == blk_of[t[:, :1]]).all()


def test_galerkin_blocks_and_restriction(scene_and_cage):
    sc, cage = scene_and_cage
    emb, t, w = _weights(cage)
    starts = np.nonzero(np.r_[True, np.diff(cage.blk_base) != 0])[0]
    rng = np.random.default_rng(0)
    xc = cage.coarse_pos.astype(np.float64) + rng.normal(scale=1e-3, size=cage.coarse_pos.shape)
    xf = (w[:, :, None] * xc[t]).sum(1)  # a fine state the cage represents exactly
    b = np.zeros_like(xc)
    for k in range(4):
        np.add.at(b, t[:, k], w[:, k:k + 1] * (xf - (w[:, :, None] * xc[t]).sum(1)))
    assert np.abs(b).max() < 1e-12  # zero residual: P^T (x - P x_c) = 0
    for s0 in starts:
        base, dim, off = int(cage.blk_base[s0]), int(cage.blk_dim[s0]), int(cage.blk_matoff[s0])
        M = cage.minv_flat[off:off + dim * dim].astype(np.float64).reshape(dim, dim)
        assert np.abs(M - M.T).max() <= 1e-6 * np.abs(M).max()
        ev = np.linalg.eigvalsh(0.5 * (M + M.T))
        assert ev.min() > 0
        # the Tikhonov term bounds the gain by 1 / lam
        assert ev.max() <= 1.0001 / cage.lam
