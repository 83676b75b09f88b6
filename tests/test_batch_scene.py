"""Batched instances on the host: scene generation, CSR packing, sharding,
grouped tile layout, persistent tile ranges, and the sharded oracle run
(world_size 2 over gloo) against the unsharded one."""
import os
import types

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from rlmusclev2_b200.builder import collect_raw_constraints
from rlmusclev2_b200.engine import XpbdEngine
from rlmusclev2_b200.layout import build_layout
from rlmusclev2_b200.meshgen import batch_subset, batched_box_scene, shard_instances
from rlmusclev2_b200.mg import load_config

CFG = "rlmusclev2_b200/configs/batched_256.json"


def _small(n=6, seed=3):
    return batched_box_scene(n_inst=n, seed=seed, tets_lo=800, tets_hi=4000)


def test_full_batch_sizes():
    sc = batched_box_scene()
    counts = np.diff(sc.inst_tptr)
    assert sc.n_inst == 256
    assert 3.4e6 < sc.tets.shape[0] < 3.6e6
    assert counts.min() >= 1500 and counts.max() <= 66000
    # log-uniform: about a quarter of the draws below the geometric quartile point
    q = np.exp(np.log(2000) + 0.25 * (np.log(60000) - np.log(2000)))
    assert 0.15 < (counts < q).mean() < 0.35
    assert (np.diff(sc.inst_vptr) > 0).all()
    v_of_t = sc.vert_inst[sc.tets]
    assert (v_of_t == sc.tet_inst[:, None]).all()


def test_small_batch_structure():
    sc = _small()
    assert sc.bone_center.shape[0] == 2 * sc.n_inst
    assert set(np.unique(sc.vert_bone[sc.inst_vptr[2]:sc.inst_vptr[3]])) == {4, 5}
    T = sc.bone_transforms(1)
    np.testing.assert_allclose(T[:, :, :3], np.tile(np.eye(3), (T.shape[0], 1, 1)), atol=1e-12)
    a = sc.instance_activation(9)
    np.testing.assert_allclose(a, sc.act_knots[:, 1], rtol=1e-6)
    assert sc.activation(5).shape == (sc.tets.shape[0],)


def test_shards_balanced_and_subset_consistent():
    sc = _small(n=9)
    counts = np.diff(sc.inst_tptr)
    sh = shard_instances(counts, 2)
    assert sorted(sh[0] + sh[1]) == list(range(9))
    loads = [counts[s].sum() for s in sh]
    assert abs(loads[0] - loads[1]) <= counts.max()
    sub = batch_subset(sc, sh[1])
    assert sub.n_inst == len(sh[1])
    i = sh[1][0]
    np.testing.assert_array_equal(sub.verts[:sub.inst_vptr[1]], sc.verts[sc.inst_vptr[i]:sc.inst_vptr[i + 1]])
    np.testing.assert_array_equal(sub.bone_transforms(7)[:2], sc.bone_transforms(7)[2 * i:2 * i + 2])


def test_grouped_layout_and_tile_ranges():
    sc = _small(n=7)
    cons = [{"type": "tetarapsvd", "name": "arap", "stiffness": 1e7}]
    t = collect_raw_constraints(sc.verts, sc.tets, cons).sorted_by_type()
    L = build_layout(sc.verts, sc.tets, t, tile_tets=512, vert_group=sc.vert_inst)
    assert (np.diff(L.tile_group) >= 0).all()
    grp_of_tet = sc.tet_inst[L.tet_perm]
    for k in range(L.n_tiles):
        g = grp_of_tet[L.tile_tptr[k]:L.tile_tptr[k + 1]]
        assert (g == L.tile_group[k]).all()
    # vertices owned by a tile belong to its group, and no vertex is touched by two groups
    own = L.tile_own
    for k in range(L.n_tiles):
        ids = L.perm[own[k]:own[k + 1]]
        assert (sc.vert_inst[ids] == L.tile_group[k]).all()
    fake = types.SimpleNamespace(layout=L)
    ntile_grp = np.bincount(L.tile_group)
    slots = int(ntile_grp.max()) + 1
    ranges = XpbdEngine._persist_ranges(fake, slots)
    assert ranges[0][0] == 0 and ranges[-1][1] == L.n_tiles
    for (b, e), (b2, _) in zip(ranges[:-1], ranges[1:]):
        assert e == b2
    for b, e in ranges:
        assert e - b <= slots
        assert b == 0 or L.tile_group[b] != L.tile_group[b - 1]
    assert XpbdEngine._persist_ranges(fake, int(ntile_grp.max()) - 1) == []


def _oracle_frames(cfg, sc, frames):
    o = O.OracleBatchSim(cfg, sc, prec="f32")
    for f in frames:
        o.step_frame(f)
    return o.pos.copy()


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg = load_config(CFG)
    cfg["demo"]["collision"]["sdf_res"] = 24
    sc = _small(n=5, seed=11)
    mine = shard_instances(np.diff(sc.inst_tptr), world)[rank]
    pos = _oracle_frames(cfg, batch_subset(sc, mine), (1, 2))
    got = [None] * world
    dist.all_gather_object(got, (mine, pos))
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_oracle_matches_unsharded_gloo():
    """Instances are independent: two gloo ranks stepping their shards give the
    same positions, bit for bit, as one process stepping the whole batch."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    cfg = load_config(CFG)
    cfg["demo"]["collision"]["sdf_res"] = 24
    sc = _small(n=5, seed=11)
    full = _oracle_frames(cfg, sc, (1, 2))
    for mine, pos in got:
        rows = np.concatenate([np.arange(sc.inst_vptr[i], sc.inst_vptr[i + 1]) for i in mine])
        np.testing.assert_array_equal(pos, full[rows])


def test_cage_lattice_neighbours():
    """The learned warm start's cage description: six axis neighbours found in
    each muscle's lattice, symmetric (+x of j has j as -x), same owner."""
    from rlmusclev2_b200.learned import cage_static
    from rlmusclev2_b200.meshgen import build_cage, humanv2_scene
    sc = humanv2_scene(seed=1, n_muscles=5, n_bones=4, target_tets=20000, fascia_tets=3000, box=(0.35, 0.35, 0.35))
    cage = build_cage(sc)
    st = cage_static(cage, sc)
    nbr = st["nbr"]
    assert (nbr >= 0).mean() > 0.5
    for q in range(6):
        j = np.nonzero(nbr[:, q] >= 0)[0]
        k = nbr[j, q]
        assert (nbr[k, q ^ 1] == j).all()
        assert (st["owner"][k] == st["owner"][j]).all()
    assert st["stat"].shape == (cage.coarse_pos.shape[0], 24)
