"""Forest (batched problems) on the CPU: the merged tree and traversal give,
through the FP64 oracle, exactly the per-problem results; lists never cross
problems and still cover every pair of leaves once; the fixed root box; the
autotuner's cache logic."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from sumpy_b200 import autotune
from sumpy_b200.forest import build_forest
from sumpy_b200.tree import build_all

BOX = [[0.0, 1.0]] * 3


def _problems(seed, P, lo=150, hi=2500):
    rng = np.random.default_rng(seed)
    return [rng.random((3, int(n))) for n in rng.integers(lo, hi, P)], rng


@pytest.mark.parametrize("separate_targets", [False, True])
def test_forest_oracle_equals_per_problem(separate_targets):
    srcs, rng = _problems(11, 6)
    tgts = [rng.random((3, int(n))) for n in rng.integers(100, 900, len(srcs))] \
        if separate_targets else None
    tree, trav, tcls, forest = build_forest(srcs, tgts, 24, bbox=BOX)
    ws = [rng.standard_normal(s.shape[1]) for s in srcs]
    order = 5
    pot = O.run_fmm(tree, trav, tcls, order, np.concatenate(ws),
                    exclude_self=not separate_targets)
    parts = forest.split_targets(pot)
    assert len(parts) == len(srcs)
    for i in range(len(srcs)):
        t, tr, tc = build_all(srcs[i], None if tgts is None else tgts[i], 24, bbox=BOX)
        ref = O.run_fmm(t, tr, tc, order, ws[i], exclude_self=not separate_targets)
        np.testing.assert_allclose(parts[i], ref, rtol=0, atol=1e-14 * np.abs(ref).max())


def _ancestors(tree, b):
    out = [int(b)]
    while tree.box_levels[b] > 0:
        b = tree.box_parent_ids[b]
        out.append(int(b))
    return out


def test_forest_lists_cover_pairs_within_each_problem():
    srcs, _ = _problems(5, 4, 300, 1500)
    tree, trav, _, forest = build_forest(srcs, None, 12, bbox=BOX)
    owner = np.full(tree.nboxes, -1)
    for i, m in enumerate(forest.box_maps):
        owner[m] = i
    assert (owner >= 0).all()
    tpos = {int(b): i for i, b in enumerate(trav.target_or_target_parent_boxes)}
    l3 = {}
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        for i, t in enumerate(tbs):
            l3.setdefault(int(t), set()).update(
                csr.lists[csr.starts[i]:csr.starts[i + 1]].tolist())
    ns, nl = trav.neighbor_source_boxes_starts, trav.neighbor_source_boxes_lists
    bad = 0
    for i, t in enumerate(trav.target_boxes):
        L1 = set(nl[ns[i]:ns[i + 1]].tolist())
        L3 = l3.get(int(t), set())
        L2, L4 = set(), set()
        for b in _ancestors(tree, t):
            j = tpos[b]
            L2 |= set(trav.from_sep_siblings_lists[
                trav.from_sep_siblings_starts[j]:trav.from_sep_siblings_starts[j + 1]].tolist())
            L4 |= set(trav.from_sep_bigger_lists[
                trav.from_sep_bigger_starts[j]:trav.from_sep_bigger_starts[j + 1]].tolist())
        for lst in (L1, L2, L3, L4):
            assert all(owner[s] == owner[t] for s in lst)
        for s in trav.source_boxes:
            if owner[s] != owner[t]:
                continue
            sa = set(_ancestors(tree, s))
            c = (int(s) in L1) + len(sa & L3) + len(sa & L2) + (int(s) in L4)
            bad += c != 1
    assert bad == 0


def test_forest_layout():
    srcs, _ = _problems(2, 5)
    tree, trav, tcls, forest = build_forest(srcs, None, 20, bbox=BOX)
    assert tree.root_extent == 1.0
    ls = tree.level_start_box_nrs
    assert ls[1] == len(srcs)                      # one root per problem
    assert (np.diff(tree.box_levels) >= 0).all()   # level-major numbering
    for lev in range(tree.nlevels):
        assert (tree.box_levels[ls[lev]:ls[lev + 1]] == lev).all()
    assert forest.source_starts[-1] == tree.nsources == sum(s.shape[1] for s in srcs)
    # particles of problem i stay in its own range
    for i, m in enumerate(forest.box_maps):
        a, b = forest.source_starts[i], forest.source_starts[i + 1]
        st = tree.box_source_starts[m]
        assert ((st >= a) & (st + tree.box_source_counts_cumul[m] <= b)).all()
    np.testing.assert_array_equal(np.sort(tree.user_source_ids), np.arange(tree.nsources))


def test_fixed_root_box():
    rng = np.random.default_rng(0)
    pts = rng.random((3, 500)) * 0.5
    tree, _, _ = build_all(pts, None, 10, bbox=BOX)
    assert tree.root_extent == 1.0
    np.testing.assert_array_equal(tree.bounding_box[0], [0, 0, 0])
    with pytest.raises(ValueError, match="outside"):
        build_all(pts + 0.8, None, 10, bbox=BOX)
    with pytest.raises(ValueError):
        build_all(pts, None, 10, bbox=[[0, 0]] * 3)


def test_forest_rejects_mixed_root_boxes():
    from sumpy_b200.forest import merge_trees
    rng = np.random.default_rng(1)
    a = build_all(rng.random((3, 100)), None, 10, bbox=BOX)
    b = build_all(rng.random((3, 100)), None, 10)
    with pytest.raises(ValueError, match="root box"):
        merge_trees([a, b])


def test_autotune_cache(tmp_path):
    path = tmp_path / "tune.json"
    calls = []

    def measure(c):
        calls.append(c)
        return {16: 3.0, 32: 1.0, 64: 2.0}[c]

    assert autotune.tune("k", [16, 32, 64], measure, path) == 32
    assert calls == [16, 32, 64]
    data = json.loads(path.read_text())
    assert data["k"]["best"] == 32
    # a cached key is not measured again
    assert autotune.tune("k", [16, 32, 64], measure, path) == 32
    assert calls == [16, 32, 64]
    # a cached best outside the candidate set is re-tuned
    assert autotune.tune("k", [16, 64], measure, path) == 64
    assert autotune.tune("k", [16, 64], measure, path, refresh=True) == 64
    assert len(calls) == 7
