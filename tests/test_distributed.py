"""The distributed FMM's host logic without a GPU: the leaf partition, the
local traversals (each rank's interaction lists restricted to its leaves and
their ancestors), and the decomposition they give -- the ranks' partial
multipoles sum to the global multipoles, and the ranks' potentials, each on
its own targets, sum to the global potentials (FP64 oracle runs over the
restricted traversals, as in sumpy/test/test_distributed.py:107-146, which
compares a distributed run with a single-rank one). A two-rank gloo run
sends the tree from the root, partitions on every rank and exchanges the
multipoles and potentials through the same collectives the GPU wrangler
uses."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from sumpy_b200 import distributed as D
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer, uniform_cube

ORDER = 5


def _problem(kind="self"):
    if kind == "self":
        src = sphere_plummer(6000, 21)
        return src, None, np.random.default_rng(5).standard_normal(6000), 20
    return uniform_cube(4000, 22), uniform_cube(3000, 23), \
        np.random.default_rng(6).standard_normal(4000), 24


def _rows(starts, lists, i):
    return np.asarray(lists)[int(starts[i]):int(starts[i + 1])]


@pytest.mark.parametrize("nranks", [1, 2, 5])
def test_partition_covers_leaves_in_morton_ranges(nranks):
    src, tgt, q, mpb = _problem()
    tree, trav, tcls = build_all(src, tgt, mpb)
    owner = D.partition_boxes(tree, trav, nranks)
    leaves = D.leaf_boxes(tree)
    assert (owner[leaves] >= 0).all() and (owner[leaves] < nranks).all()
    nonleaf = np.setdiff1d(np.arange(tree.nboxes), leaves)
    assert (owner[nonleaf] == -1).all()
    order = leaves[np.argsort(D.morton_keys(tree, leaves), kind="stable")]
    assert (np.diff(owner[order]) >= 0).all()             # contiguous ranges
    cost = D.leaf_costs(tree, trav)
    share = np.array([cost[owner == r].sum() for r in range(nranks)]) / cost.sum()
    assert share.max() < 1.0 / nranks + cost.max() / cost.sum() + 1e-12


def test_morton_keys_are_unique_and_ordered_within_parents():
    tree, trav, tcls = build_all(uniform_cube(3000, 2), None, 10)
    leaves = D.leaf_boxes(tree)
    keys = D.morton_keys(tree, leaves)
    assert len(np.unique(keys)) == len(leaves)


@pytest.mark.parametrize("kind", ["self", "separate"])
def test_local_traversals_partition_the_lists(kind):
    src, tgt, q, mpb = _problem(kind)
    tree, trav, tcls = build_all(src, tgt, mpb)
    R = 3
    owner = D.partition_boxes(tree, trav, R)
    locs = [D.local_traversal(tree, trav, tcls, owner, r) for r in range(R)]
    # leaves: sources and targets split without overlap
    for name in ("source_boxes", "target_boxes"):
        parts = [np.asarray(getattr(lt, name)) for lt, _ in locs]
        allp = np.concatenate(parts)
        assert len(allp) == len(np.unique(allp)) == len(getattr(trav, name))
        assert set(allp) == set(np.asarray(getattr(trav, name)))
    # List 1 and List 3 rows are the global rows of the owned targets
    g1 = {int(b): _rows(trav.neighbor_source_boxes_starts, trav.neighbor_source_boxes_lists, i)
          for i, b in enumerate(trav.target_boxes)}
    for lt, _ in locs:
        for i, b in enumerate(lt.target_boxes):
            assert np.array_equal(_rows(lt.neighbor_source_boxes_starts,
                                        lt.neighbor_source_boxes_lists, i), g1[int(b)])
        for lev, (tbs, csr) in enumerate(zip(lt.target_boxes_sep_smaller_by_source_level,
                                             lt.from_sep_smaller_by_level)):
            gt = np.asarray(trav.target_boxes_sep_smaller_by_source_level[lev])
            gc = trav.from_sep_smaller_by_level[lev]
            pos = {int(b): i for i, b in enumerate(gt)}
            for i, b in enumerate(tbs):
                assert np.array_equal(_rows(csr.starts, csr.lists, i),
                                      _rows(gc.starts, gc.lists, pos[int(b)]))
    n3 = sum(len(c.lists) for lt, _ in locs for c in lt.from_sep_smaller_by_level)
    assert n3 == sum(len(c.lists) for c in trav.from_sep_smaller_by_level)
    # Lists 2 and 4: every global row kept by some rank, rows and classes unchanged
    ttp = np.asarray(trav.target_or_target_parent_boxes)
    pos = {int(b): i for i, b in enumerate(ttp)}
    covered = set()
    for lt, lc in locs:
        for i, b in enumerate(lt.target_or_target_parent_boxes):
            gi = pos[int(b)]
            covered.add(int(b))
            assert np.array_equal(_rows(lt.from_sep_siblings_starts, lt.from_sep_siblings_lists, i),
                                  _rows(trav.from_sep_siblings_starts,
                                        trav.from_sep_siblings_lists, gi))
            assert np.array_equal(
                _rows(lt.from_sep_siblings_starts, lc.from_sep_siblings_translation_classes, i),
                _rows(trav.from_sep_siblings_starts, tcls.from_sep_siblings_translation_classes,
                      gi))
            assert np.array_equal(_rows(lt.from_sep_bigger_starts, lt.from_sep_bigger_lists, i),
                                  _rows(trav.from_sep_bigger_starts, trav.from_sep_bigger_lists,
                                        gi))
        ls = np.asarray(lt.level_start_target_or_target_parent_box_nrs)
        levs = np.asarray(tree.box_levels)[np.asarray(lt.target_or_target_parent_boxes)]
        for lev in range(tree.nlevels):
            assert (levs[ls[lev]:ls[lev + 1]] == lev).all()
    assert covered == set(ttp.tolist())


@pytest.mark.parametrize("kind", ["self", "separate"])
def test_ranks_sum_to_the_global_fmm(kind):
    """Oracle FMM over each rank's traversal: partial multipoles and
    own-target potentials add up to the single-rank FMM."""
    src, tgt, q, mpb = _problem(kind)
    tree, trav, tcls = build_all(src, tgt, mpb)
    excl = tgt is None
    ref_st = {}
    ref = O.run_fmm(tree, trav, tcls, ORDER, q, exclude_self=excl, stages=ref_st)
    R = 3
    owner = D.partition_boxes(tree, trav, R)
    msum = np.zeros_like(ref_st["mpoles"])
    psum = np.zeros_like(ref)
    for r in range(R):
        lt, lc = D.local_traversal(tree, trav, tcls, owner, r)
        st = {}
        O.run_fmm(tree, lt, lc, ORDER, q, exclude_self=excl, stages=st)
        msum += st["mpoles"]
        # the downward pass of this rank on the global multipoles
        lt2, lc2 = D.local_traversal(tree, trav, tcls, owner, r, restrict_sources=False)
        pr = O.run_fmm(tree, lt2, lc2, ORDER, q, exclude_self=excl)
        # user index of each tree-ordered target (potentials come back as
        # tree_pot[sorted_target_ids])
        sti = np.asarray(tree.sorted_target_ids)
        user_of = np.empty_like(sti)
        user_of[sti] = np.arange(len(sti))
        mine = np.zeros(tree.ntargets, dtype=bool)
        for b in np.asarray(lt2.target_boxes):
            s0 = int(tree.box_target_starts[b])
            mine[user_of[s0:s0 + int(tree.box_target_counts_nonchild[b])]] = True
        assert np.all(pr[~mine] == 0.0)
        psum += pr
    assert np.linalg.norm(msum - ref_st["mpoles"]) <= 1e-13 * np.linalg.norm(ref_st["mpoles"])
    assert np.linalg.norm(psum - ref) <= 1e-13 * np.linalg.norm(ref)


def test_tree_pack_roundtrip():
    src, tgt, q, mpb = _problem("separate")
    tree, trav, tcls = build_all(src, tgt, mpb)
    t2, v2, c2 = D.unpack_tree(D.pack_tree(tree, trav, tcls))
    assert t2.nboxes == tree.nboxes and np.array_equal(t2.box_centers, tree.box_centers)
    assert np.array_equal(v2.from_sep_siblings_lists, trav.from_sep_siblings_lists)
    assert np.array_equal(c2.from_sep_siblings_translation_classes,
                          tcls.from_sep_siblings_translation_classes)
    assert t2._traversal is v2 and v2.tree is t2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        src, tgt, q, mpb = _problem("self")
        tree0 = build_all(src, tgt, mpb)[0] if rank == 0 else None
        tree, trav, tcls = D.broadcast_tree(tree0)
        owner = D.partition_boxes(tree, trav, world)
        lt, lc = D.local_traversal(tree, trav, tcls, owner, rank)
        st = {}
        O.run_fmm(tree, lt, lc, ORDER, q, exclude_self=True, stages=st)
        mp_ = torch.as_tensor(st["mpoles"])
        D.allreduce_sum_(mp_)                       # the exchange step
        lt2, lc2 = D.local_traversal(tree, trav, tcls, owner, rank, restrict_sources=False)
        pot = torch.as_tensor(O.run_fmm(tree, lt2, lc2, ORDER, q, exclude_self=True))
        D.reduce_sum_to_root_(pot)
        qw = torch.as_tensor(q if rank == 0 else np.zeros_like(q))
        D.broadcast_(qw)
        if rank == 0:
            out_q.put((mp_.numpy(), pot.numpy(), owner, qw.numpy()))
        else:
            out_q.put(("owner", owner, float(qw.sum())))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_distributed_fmm_host_path():
    ctx = mp.get_context("spawn")
    qq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, qq)) for r in range(2)]
    for p in procs:
        p.start()
    got = [qq.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    root = next(g for g in got if not isinstance(g[0], str))
    other = next(g for g in got if isinstance(g[0], str))
    mpoles, pot, owner0, qw = root
    src, tgt, q, mpb = _problem("self")
    tree, trav, tcls = build_all(src, tgt, mpb)
    st = {}
    ref = O.run_fmm(tree, trav, tcls, ORDER, q, exclude_self=True, stages=st)
    assert np.array_equal(owner0, other[1])                  # same partition on both ranks
    assert np.array_equal(qw, q) and other[2] == pytest.approx(float(q.sum()))
    assert np.linalg.norm(mpoles - st["mpoles"]) <= 1e-13 * np.linalg.norm(st["mpoles"])
    assert np.linalg.norm(pot - ref) <= 1e-13 * np.linalg.norm(ref)
