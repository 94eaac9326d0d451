"""Tree/traversal invariants (boxtree's role; its lists are not pinned by any
reference test, so they are checked by the covering property of the FMM:
every (target box, source box) pair of leaves is handled exactly once by
List 1, List 3, or List 2 / List 4 of an ancestor-or-self of the target)."""
import numpy as np
import pytest

from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer


def _anc(par, b):
    out = [int(b)]
    while b != 0:
        b = par[b]
        out.append(int(b))
    return out


def coverage_violations(tree, trav):
    par = tree.box_parent_ids
    tpos = {int(b): i for i, b in enumerate(trav.target_or_target_parent_boxes)}
    l3 = {}
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        for i, t in enumerate(tbs):
            l3.setdefault(int(t), set()).update(csr.lists[csr.starts[i]:csr.starts[i + 1]].tolist())
    bad = 0
    ns = trav.neighbor_source_boxes_starts
    nl = trav.neighbor_source_boxes_lists
    for i, t in enumerate(trav.target_boxes):
        L1 = set(nl[ns[i]:ns[i + 1]].tolist())
        L3 = l3.get(int(t), set())
        L2, L4 = set(), set()
        for b in _anc(par, t):
            j = tpos[b]
            L2 |= set(trav.from_sep_siblings_lists[
                trav.from_sep_siblings_starts[j]:trav.from_sep_siblings_starts[j + 1]].tolist())
            L4 |= set(trav.from_sep_bigger_lists[
                trav.from_sep_bigger_starts[j]:trav.from_sep_bigger_starts[j + 1]].tolist())
        for s in trav.source_boxes:
            sa = set(_anc(par, s))
            c = (int(s) in L1) + len(sa & L3) + len(sa & L2) + (int(s) in L4)
            bad += c != 1
    return bad


@pytest.mark.parametrize("kind", ["sphere_plummer", "separate_targets", "uniform"])
def test_lists_cover_every_pair_once(kind):
    rng = np.random.default_rng(3)
    if kind == "sphere_plummer":
        tree, trav, _ = build_all(sphere_plummer(2500, 7), None, 8)
    elif kind == "separate_targets":
        tree, trav, _ = build_all(rng.standard_normal((3, 1200)),
                                  rng.standard_normal((3, 600)) * 0.5 + 0.3, 5)
    else:
        tree, trav, _ = build_all(rng.random((3, 3000)), rng.random((3, 1000)), 30)
    assert coverage_violations(tree, trav) == 0
    if kind != "uniform":
        assert sum(len(x.lists) for x in trav.from_sep_smaller_by_level) > 0
        assert len(trav.from_sep_bigger_lists) > 0


def test_tree_fields():
    rng = np.random.default_rng(1)
    src = rng.random((3, 5000))
    tgt = rng.random((3, 3000))
    tree, trav, tcls = build_all(src, tgt, 30)
    # particles sorted into boxes; permutations
    assert np.allclose(tree.sources, src[:, tree.user_source_ids])
    assert np.allclose(tree.targets[:, tree.sorted_target_ids], tgt)
    for b in range(tree.nboxes):
        s0, n = tree.box_source_starts[b], tree.box_source_counts_cumul[b]
        h = tree.root_extent * 2.0 ** -tree.box_levels[b]
        pts = tree.sources[:, s0:s0 + n]
        assert np.all(np.abs(pts - tree.box_centers[:, b:b + 1]) <= h / 2 * (1 + 1e-12))
    # refinement rule
    leaves = np.all(tree.box_child_ids == 0, axis=0)
    tot = tree.box_source_counts_cumul + tree.box_target_counts_cumul
    assert np.all(tot[~leaves] > 30)
    # level-ordered boxes
    assert np.all(np.diff(tree.box_levels) >= 0)
    lev = tree.box_levels
    for L in range(tree.nlevels):
        a, b = tree.level_start_box_nrs[L:L + 2]
        assert np.all(lev[a:b] == L)
    # translation classes: 316 per level >= 2; vector = target - source center
    ls = tcls.from_sep_siblings_translation_classes_level_starts
    assert all(ls[L + 1] - ls[L] == (316 if L >= 2 else 0) for L in range(tree.nlevels))
    cv = tcls.from_sep_siblings_translation_class_to_distance_vector
    st = trav.from_sep_siblings_starts
    for j, t in enumerate(trav.target_or_target_parent_boxes[:200]):
        for e in range(st[j], st[j + 1]):
            s = trav.from_sep_siblings_lists[e]
            c = tcls.from_sep_siblings_translation_classes[e]
            assert np.allclose(cv[:, c], tree.box_centers[:, t] - tree.box_centers[:, s])


def test_edge_cases():
    # a single box (fewer particles than the limit)
    tree, trav, _ = build_all(np.random.default_rng(0).random((3, 10)), None, 30)
    assert tree.nboxes == 1 and tree.nlevels == 1
    assert list(trav.target_boxes) == [0]
    assert len(trav.from_sep_siblings_lists) == 0
    # duplicated points stop refining at the level cap
    pts = np.zeros((3, 50)) + 0.5
    pts[:, :5] = np.random.default_rng(0).random((3, 5))
    tree, trav, _ = build_all(pts, None, 10, max_levels=6)
    assert tree.nlevels <= 6
    assert coverage_violations(tree, trav) == 0
    # empty source set with targets
    tree, trav, _ = build_all(np.zeros((3, 0)), np.random.default_rng(0).random((3, 40)), 8)
    assert tree.nsources == 0 and len(trav.source_boxes) == 0
    with pytest.raises(ValueError):
        build_all(np.array([[0.0, np.nan], [0, 0], [0, 0]]), None, 4)
