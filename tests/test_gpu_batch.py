"""Batched evaluation on the GPU: a forest of problems through one
``drive_fmm`` (eager and replayed as a CUDA graph) against each problem run
on its own, the mixed form against the FP64 form, and the autotuner."""
import numpy as np
import pytest
import torch

from sumpy_b200 import (
    LaplaceKernel,
    LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
    LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp,
    SumpyExpansionWrangler,
    SumpyTreeIndependentDataForWrangler,
    drive_fmm,
)
from sumpy_b200.batch import BatchedLaplaceFMM
from sumpy_b200.tree import build_all

pytestmark = pytest.mark.gpu

BOX = [[0.0, 1.0]] * 3


def _rel(a, b):
    a, b = torch.as_tensor(a).cpu().numpy(), torch.as_tensor(b).cpu().numpy()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _problems(seed, P):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(300), np.log(6000), P)).astype(int)
    return [rng.random((3, int(k))) for k in n], rng


def _single(src, w, order, dev):
    tree, trav, tcls = build_all(src, None, 32, bbox=BOX)
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(None, lambda o: MExp(knl, o),
                                             lambda o: LExp(knl, o), [knl], exclude_self=True)
    wr = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                                translation_classes_data=tcls, device=dev)
    (pot,) = drive_fmm(None, wr, [torch.as_tensor(w, device=dev)])
    return pot


def test_batch_matches_single_problems(cuda_device):
    srcs, rng = _problems(3, 12)
    ws = [rng.standard_normal(s.shape[1]) for s in srcs]
    order = 6
    b = BatchedLaplaceFMM(srcs, order=order, precision="fp64", bbox=BOX, device=cuda_device,
                          use_graph=False)
    parts = b(ws)
    for i in (0, 5, 11):
        ref = _single(srcs[i], ws[i], order, cuda_device)
        assert _rel(parts[i], ref) < 1e-12


def test_graph_replay_matches_eager(cuda_device):
    srcs, rng = _problems(4, 16)
    eager = BatchedLaplaceFMM(srcs, order=8, precision="mixed", bbox=BOX, device=cuda_device,
                              use_graph=False)
    graphed = BatchedLaplaceFMM(srcs, order=8, precision="mixed", bbox=BOX,
                                device=cuda_device, use_graph=True)
    for _ in range(2):     # new strengths each call: the graph reads its input buffer
        w = torch.as_tensor(rng.standard_normal(eager.nsources))
        a = eager.evaluate(w)
        g = graphed.evaluate(w)
        assert _rel(g, a) < 1e-12
    graphed.check_status()


def test_batch_mixed_within_tolerance_of_fp64(cuda_device):
    srcs, rng = _problems(5, 10)
    w = rng.standard_normal(sum(s.shape[1] for s in srcs))
    f = BatchedLaplaceFMM(srcs, order=8, precision="fp64", bbox=BOX, device=cuda_device)
    m = BatchedLaplaceFMM(srcs, order=8, precision="mixed", bbox=BOX, device=cuda_device)
    assert _rel(m.evaluate(w), f.evaluate(w)) < 2e-6


def test_autotune_picks_and_caches(cuda_device, tmp_path):
    """The schedule autotuner searches the knobs, stores the best schedule,
    and a second batch of the same shape takes it from the cache; any
    schedule gives the same FP64 result."""
    import json
    from sumpy_b200.autotune import SCHEDULE_SPACE
    srcs, rng = _problems(6, 8)
    path = tmp_path / "tune.json"
    b = BatchedLaplaceFMM(srcs, order=6, precision="fp64", bbox=BOX, device=cuda_device,
                          autotune=True, autotune_cache=path)
    for k, v in b.schedule.items():
        assert v in SCHEDULE_SPACE[k]
    assert path.exists()
    entry = next(iter(json.loads(path.read_text()).values()))
    assert entry["best"] == b.schedule and len(entry["tried"]) >= len(SCHEDULE_SPACE)
    b2 = BatchedLaplaceFMM(srcs, order=6, precision="fp64", bbox=BOX, device=cuda_device,
                           autotune=True, autotune_cache=path)
    assert b2.schedule == b.schedule
    w = torch.as_tensor(rng.standard_normal(b.nsources))
    ref = BatchedLaplaceFMM(srcs, order=6, precision="fp64", bbox=BOX, device=cuda_device,
                            use_graph=False, m2l_item_groups=64).evaluate(w)
    assert _rel(b.evaluate(w), ref) < 1e-12
    b.check_status()
