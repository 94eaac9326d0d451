"""Host-side work items of the one-launch M2P and P2L kernels
(sumpy_b200.fmm.m2p_items / p2l_items): every (target, List-3 box) pair and
every (target box, List-4 source) pair of the traversal is covered exactly
once, items respect the kernels' limits (32 targets, lane groups, rounds),
carry the right level, and come longest first."""
import numpy as np
import pytest

from sumpy_b200.fmm import ITEM_ROUNDS, M2P_ITEM_GROUPS, m2p_items, p2l_items
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer


@pytest.fixture(scope="module", params=[16, 96])
def traversal(request):
    pts = sphere_plummer(30000, 3)
    return build_all(pts, None, request.param)


def _lane_groups(ntc, groups=M2P_ITEM_GROUPS):
    g = 32 // groups
    while g < ntc:
        g *= 2
    return 32 // g


# M2P_ITEM_GROUPS: the mixed kernel (FP32 multipoles staged per lane group);
# 32: the FP64 and Helmholtz kernels (lane groups from one lane)
@pytest.mark.parametrize("groups", [M2P_ITEM_GROUPS, 32])
def test_m2p_items_cover_list3_once(traversal, groups):
    tree, trav, _ = traversal
    items, lists = m2p_items(tree, trav.target_boxes_sep_smaller_by_source_level,
                             trav.from_sep_smaller_by_level, groups=groups)
    assert items.dtype == np.int32 and items.flags.c_contiguous and items.shape[1] == 4
    # expected (target, global list entry) pairs and each entry's level
    want, entry_level, off = [], [], 0
    for lev, (tbs, csr) in enumerate(zip(trav.target_boxes_sep_smaller_by_source_level,
                                         trav.from_sep_smaller_by_level)):
        st = np.asarray(csr.starts)
        entry_level += [lev] * len(csr.lists)
        for i, tb in enumerate(np.asarray(tbs)):
            t0, nt = tree.box_target_starts[tb], tree.box_target_counts_nonchild[tb]
            for e in range(st[i], st[i + 1]):
                want += [(t, off + e) for t in range(t0, t0 + nt)]
        off += len(csr.lists)
    np.testing.assert_array_equal(lists, np.concatenate(
        [np.asarray(c.lists) for c in trav.from_sep_smaller_by_level]))
    got, cost = [], []
    for t0, l0, nb, w in items:
        ntc, lev = w & 0xff, w >> 8
        nph = _lane_groups(ntc, groups)
        assert 1 <= ntc <= 32 and 1 <= nb <= nph * ITEM_ROUNDS
        assert all(entry_level[e] == lev for e in range(l0, l0 + nb))
        got += [(t, e) for t in range(t0, t0 + ntc) for e in range(l0, l0 + nb)]
        cost.append(-(-nb // nph))
    assert len(got) == len(want) > 0
    assert sorted(got) == sorted(want)
    assert all(a >= b for a, b in zip(cost, cost[1:]))


def test_p2l_items_cover_list4_once(traversal):
    tree, trav, _ = traversal
    lt = trav.level_start_target_or_target_parent_box_nrs
    tb_all = trav.target_or_target_parent_boxes
    st, ls = trav.from_sep_bigger_starts, trav.from_sep_bigger_lists
    items, sidx = p2l_items(tree, lt, tb_all, st, ls)
    assert items.dtype == np.int32 and items.shape[1] == 4
    want = []
    for i, tb in enumerate(tb_all):
        for sb in ls[st[i]:st[i + 1]]:
            s0 = tree.box_source_starts[sb]
            want += [(int(tb), s) for s in range(s0, s0 + tree.box_source_counts_nonchild[sb])]
    got = []
    for tb, f0, c, lev in items:
        assert 1 <= c <= 32 * ITEM_ROUNDS
        assert tree.box_levels[tb] == lev
        got += [(int(tb), int(s)) for s in sidx[f0:f0 + c]]
    assert len(got) == len(want) > 0
    assert sorted(got) == sorted(want)
    assert all(a >= b for a, b in zip(items[:, 2], items[1:, 2]))


def test_items_of_empty_lists():
    pts = sphere_plummer(200, 1)
    tree, trav, _ = build_all(pts, None, 400)   # a single box: no List 3 / List 4
    items, _ = m2p_items(tree, trav.target_boxes_sep_smaller_by_source_level,
                         trav.from_sep_smaller_by_level)
    assert items.shape == (0, 4)
    items, sidx = p2l_items(tree, trav.level_start_target_or_target_parent_box_nrs,
                            trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                            trav.from_sep_bigger_lists)
    assert items.shape == (0, 4) and sidx.size == 0


def test_l2p_packing_covers_targets_once(traversal):
    from sumpy_b200.fmm import L2P_ITEM_SLOTS, l2p_items
    tree, trav, _ = traversal
    items, slots = l2p_items(tree, trav.level_start_target_box_nrs, trav.target_boxes)
    assert items.dtype == np.int32 and items.shape[1] == 2 and slots.shape[1] == 4
    seen = np.zeros(tree.ntargets, dtype=np.int64)
    lev_of = {}
    for lev in range(tree.nlevels):
        a, b = trav.level_start_target_box_nrs[lev:lev + 2]
        for tb in trav.target_boxes[a:b]:
            lev_of[int(tb)] = lev
    for first, n in items:
        assert 1 <= n <= L2P_ITEM_SLOTS
        sl = slots[first:first + n]
        assert sl[:, 2].sum() <= 32 and (sl[:, 2] >= 1).all()
        for box, t0, cnt, lev in sl:
            assert lev == lev_of[int(box)] == tree.box_levels[box]
            assert tree.box_target_starts[box] <= t0
            assert t0 + cnt <= tree.box_target_starts[box] + tree.box_target_counts_nonchild[box]
            seen[t0:t0 + cnt] += 1
    # every target of a target box exactly once (the slots tile each box)
    want = np.zeros(tree.ntargets, dtype=np.int64)
    for tb in trav.target_boxes:
        t0 = tree.box_target_starts[tb]
        want[t0:t0 + tree.box_target_counts_nonchild[tb]] = 1
    np.testing.assert_array_equal(seen, want)
    # packing is dense: slots cover all items contiguously, and next fit
    # closes an item only when it is full (32 targets or L2P_ITEM_SLOTS
    # slots) or the next slot would not fit
    assert items[0, 0] == 0 and (items[1:, 0] == np.cumsum(items[:, 1])[:-1]).all()
    ntg = np.array([slots[f:f + n, 2].sum() for f, n in items])
    for i in range(len(items) - 1):
        nxt = slots[items[i + 1, 0], 2]
        assert ntg[i] == 32 or items[i, 1] == L2P_ITEM_SLOTS or ntg[i] + nxt > 32, i
    assert want.sum() / (32 * len(items)) > 0.5
