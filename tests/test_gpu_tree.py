"""The GPU tree / traversal / translation-class builder against the host
builder: every array bit for bit (sources, boxes, Lists 1-4, List 3 by
level, translation classes), for single trees and for forests of
independent problems (against per-problem host trees merged by
``merge_trees``), plus the covering invariant of the interaction lists."""
import numpy as np
import pytest
import torch

from sumpy_b200.forest import build_forest
from sumpy_b200.tree import build_all, build_all_gpu
from tests._pointsets import sphere_plummer, uniform_cube
from tests.test_tree import coverage_violations

pytestmark = pytest.mark.gpu

TREE_FIELDS = [
    "nsources", "ntargets", "nboxes", "nlevels", "sources_are_targets", "root_extent",
    "sources", "targets", "user_source_ids", "sorted_target_ids", "level_start_box_nrs",
    "box_centers", "box_levels", "box_parent_ids", "box_child_ids", "box_coords",
    "box_source_starts", "box_source_counts_cumul", "box_source_counts_nonchild",
    "box_target_starts", "box_target_counts_cumul", "box_target_counts_nonchild",
    "target_to_source"]
TRAV_FIELDS = [
    "source_boxes", "target_boxes", "source_parent_boxes", "target_or_target_parent_boxes",
    "level_start_source_box_nrs", "level_start_target_box_nrs",
    "level_start_source_parent_box_nrs", "level_start_target_or_target_parent_box_nrs",
    "neighbor_source_boxes_starts", "neighbor_source_boxes_lists",
    "from_sep_siblings_starts", "from_sep_siblings_lists",
    "from_sep_bigger_starts", "from_sep_bigger_lists"]
TCLS_FIELDS = [
    "from_sep_siblings_translation_classes",
    "from_sep_siblings_translation_class_to_distance_vector",
    "from_sep_siblings_translation_classes_level_starts"]


def _same(a, b, what):
    if a is None or b is None:
        assert a is None and b is None, what
        return
    if np.isscalar(a) or isinstance(a, (bool, int, float)):
        assert a == b, (what, a, b)
        return
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    assert np.array_equal(a, b), what


def assert_identical(ref, got):
    (tree0, trav0, tcls0), (tree1, trav1, tcls1) = ref, got
    for f in TREE_FIELDS:
        _same(getattr(tree0, f), getattr(tree1, f), f)
    _same(tree0.bounding_box[0], tree1.bounding_box[0], "bounding_box")
    for f in TRAV_FIELDS:
        _same(getattr(trav0, f), getattr(trav1, f), f)
    assert len(trav0.from_sep_smaller_by_level) == len(trav1.from_sep_smaller_by_level)
    for lev, (a, b) in enumerate(zip(trav0.from_sep_smaller_by_level,
                                     trav1.from_sep_smaller_by_level)):
        _same(a.starts, b.starts, f"list3 starts level {lev}")
        _same(a.lists, b.lists, f"list3 lists level {lev}")
        _same(trav0.target_boxes_sep_smaller_by_source_level[lev],
              trav1.target_boxes_sep_smaller_by_source_level[lev], f"list3 targets level {lev}")
    for f in TCLS_FIELDS:
        _same(getattr(tcls0, f), getattr(tcls1, f), f)


CASES = {
    "uniform_separate": lambda: (uniform_cube(30000, 15), uniform_cube(20000, 18), 30, None),
    "sphere_plummer_self": lambda: (sphere_plummer(60000, 7), None, 16, None),
    "clustered_deep": lambda: (np.concatenate([uniform_cube(2000, 3) * 1e-5,
                                               uniform_cube(2000, 4)], axis=1), None, 8, None),
    "clustered_small": lambda: (np.concatenate([uniform_cube(300, 3) * 1e-4,
                                                uniform_cube(300, 4)], axis=1),
                                uniform_cube(200, 6), 6, None),
    "tiny": lambda: (uniform_cube(7, 1), uniform_cube(3, 2), 30, None),
    "single_point": lambda: (np.zeros((3, 1)), None, 1, None),
    "max_levels": lambda: (sphere_plummer(20000, 9), None, 4, 5),
    "fixed_box": lambda: (uniform_cube(5000, 11) * 0.5 + 0.25, None, 12, None),
}


@pytest.mark.parametrize("case", list(CASES))
def test_gpu_tree_identical_to_host(cuda_device, case):
    src, tgt, mpb, max_levels = CASES[case]()
    bbox = [[0.0, 1.0]] * 3 if case == "fixed_box" else None
    ref = build_all(src, tgt, mpb, max_levels, bbox=bbox)
    got = build_all_gpu(src, tgt, mpb, max_levels, bbox=bbox, device=cuda_device)
    assert_identical(ref, got)
    if got[0].nboxes < 1500:     # the invariant check is quadratic in boxes
        assert coverage_violations(got[0], got[1]) == 0


def test_gpu_tree_from_device_tensors(cuda_device):
    src = sphere_plummer(40000, 3)
    ref = build_all(src, None, 24)
    got = build_all(torch.as_tensor(src, device=cuda_device), None, 24)
    assert_identical(ref, got)


def test_gpu_tree_rejects_bad_input(cuda_device):
    pts = uniform_cube(100, 5)
    pts[1, 7] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        build_all_gpu(pts, None, 10, device=cuda_device)
    with pytest.raises(ValueError, match="outside the given root box"):
        build_all_gpu(uniform_cube(100, 5) + 0.8, None, 10, bbox=[[0, 1]] * 3,
                      device=cuda_device)


@pytest.mark.parametrize("with_targets", [False, True])
def test_gpu_forest_identical_to_merged_host_trees(cuda_device, with_targets):
    rng = np.random.default_rng(3)
    sizes = [1, 40, 3000, 700, 12000, 5, 9000, 2500]
    srcs = [rng.random((3, n)) for n in sizes]
    tgts = [rng.random((3, max(1, n // 2))) for n in sizes] if with_targets else None
    box = [[0.0, 1.0]] * 3
    host = build_forest(srcs, tgts, 24, bbox=box)
    gpu = build_forest(srcs, tgts, 24, bbox=box, device=cuda_device)
    assert_identical(host[:3], gpu[:3])
    _same(host[3].source_starts, gpu[3].source_starts, "source_starts")
    _same(host[3].target_starts, gpu[3].target_starts, "target_starts")
    for i, (a, b) in enumerate(zip(host[3].box_maps, gpu[3].box_maps)):
        _same(a, b, f"box_maps[{i}]")


def test_gpu_forest_default_box(cuda_device):
    rng = np.random.default_rng(8)
    srcs = [rng.standard_normal((3, n)) for n in (500, 4000, 1200)]
    host = build_forest(srcs, None, 16)
    gpu = build_forest(srcs, None, 16, device=cuda_device)
    assert_identical(host[:3], gpu[:3])
