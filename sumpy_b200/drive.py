"""``drive_fmm``: the FMM stage sequence of boxtree's driver.

sumpy's wrangler is driven by ``boxtree.fmm.drive_fmm`` (called at
sumpy/test/test_fmm.py:280-282), which is outside the sumpy sources. This
function issues the same wrangler calls with the same traversal fields and
returns the same result (the order sumpy's wrangler documents,
sumpy/fmm.py:609-1086):

reorder_sources -> form_multipoles (P2M) -> coarsen_multipoles (M2M) ->
eval_direct (List 1) -> multipole_to_local (List 2) -> eval_multipoles
(List 3) -> form_locals (List 4) -> refine_locals (L2L) -> eval_locals (L2P)
-> reorder_potentials -> finalize_potentials.

On a CUDA wrangler the multipole/local chain (P2M, M2M, M2L, L2L, L2P) runs
on a high-priority stream and the stages that do not depend on it on a
low-priority one: List 1 and List 4 need only the strengths, List 3 only the
finished multipoles, so they fill the SMs the chain leaves idle (its coarse
levels) without delaying it. Both streams fork from the caller's stream
after the strengths are reordered and join back before the potentials are
returned; the results are ordered on the caller's stream like every other
result, and the whole sequence can be captured in a CUDA graph.
"""
from __future__ import annotations


def _side_streams(wrangler):
    """(critical, side) streams of a CUDA wrangler that allows concurrent
    stages: the multipole/local chain on a high-priority stream, the
    independent stages on a low-priority one."""
    import torch
    dev = getattr(wrangler, "device", None)
    if dev is None or getattr(dev, "type", None) != "cuda" or not getattr(
            wrangler, "concurrent_stages", False):
        return None
    s = getattr(wrangler, "_streams", None)
    if s is None:
        lo, hi = torch.cuda.Stream.priority_range()
        s = (torch.cuda.Stream(dev, priority=hi), torch.cuda.Stream(dev, priority=lo))
        wrangler._streams = s
    return s


def drive_fmm(actx, wrangler, src_weight_vecs, timing_data=None):
    if getattr(wrangler, "cuda_graph", False):
        return _drive_graphed(actx, wrangler, src_weight_vecs)
    return _drive_eager(actx, wrangler, src_weight_vecs)


def _drive_graphed(actx, wrangler, src_weight_vecs):
    """The same stage sequence replayed from a CUDA graph: captured on the
    first call (after one eager pass that builds the wrangler's plans and
    operator tables) with static copies of the strengths; every call copies
    the strengths in (host or device), replays, and returns copies of the
    static potentials. The graph is kept per input signature; it records the
    wrangler's state at capture (traversal, precision and stage switches)."""
    import torch
    dev = wrangler.device
    key = tuple((tuple(w.shape), w.dtype) for w in src_weight_vecs)
    cache = getattr(wrangler, "_graph_cache", None)
    if cache is None or cache[0] != key:
        static = [torch.empty(w.shape, dtype=w.dtype, device=dev) for w in src_weight_vecs]
        for s, w in zip(static, src_weight_vecs):
            s.copy_(w)
        cur = torch.cuda.current_stream(dev)
        warm = torch.cuda.Stream(dev)
        warm.wait_stream(cur)
        with torch.cuda.stream(warm):
            _drive_eager(actx, wrangler, static)
        cur.wait_stream(warm)
        torch.cuda.synchronize(dev)
        from sumpy_b200._capi import launch_counter
        graph = torch.cuda.CUDAGraph()
        n0 = launch_counter.value
        with torch.cuda.graph(graph):
            out = _drive_eager(actx, wrangler, static)
        # C-ABI launches recorded in the graph; each replay runs them again
        nlaunch = launch_counter.value - n0
        launch_counter.value = n0
        wrangler._graph_cache = cache = (key, graph, static, out, nlaunch)
    _, graph, static, out, nlaunch = cache
    for s, w in zip(static, src_weight_vecs):
        s.copy_(w, non_blocking=True)
    graph.replay()
    from sumpy_b200._capi import launch_counter
    launch_counter.value += nlaunch
    return [o.clone() for o in out]


def _drive_eager(actx, wrangler, src_weight_vecs):
    trav = wrangler.traversal
    src_weight_vecs = [wrangler.reorder_sources(w) for w in src_weight_vecs]
    src_weight_vecs = wrangler.distribute_source_weights(src_weight_vecs)

    streams = _side_streams(wrangler)
    if streams is not None:
        return _drive_concurrent(actx, wrangler, trav, src_weight_vecs, *streams)

    mpole_exps = wrangler.form_multipoles(
        actx, trav.level_start_source_box_nrs, trav.source_boxes, src_weight_vecs)
    mpole_exps = wrangler.coarsen_multipoles(
        actx, trav.level_start_source_parent_box_nrs, trav.source_parent_boxes, mpole_exps)
    wrangler.communicate_mpoles(actx, mpole_exps)

    potentials = wrangler.eval_direct(
        actx, trav.target_boxes, trav.neighbor_source_boxes_starts,
        trav.neighbor_source_boxes_lists, src_weight_vecs)

    local_exps = wrangler.multipole_to_local(
        actx, trav.level_start_target_or_target_parent_box_nrs,
        trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
        trav.from_sep_siblings_lists, mpole_exps)

    mpole_result = wrangler.eval_multipoles(
        actx, trav.target_boxes_sep_smaller_by_source_level,
        trav.from_sep_smaller_by_level, mpole_exps)
    potentials = [a + b for a, b in zip(potentials, mpole_result)]

    if trav.from_sep_close_smaller_starts is not None:
        direct = wrangler.eval_direct(
            actx, trav.target_boxes, trav.from_sep_close_smaller_starts,
            trav.from_sep_close_smaller_lists, src_weight_vecs)
        potentials = [a + b for a, b in zip(potentials, direct)]

    local_result = wrangler.form_locals(
        actx, trav.level_start_target_or_target_parent_box_nrs,
        trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
        trav.from_sep_bigger_lists, src_weight_vecs)
    local_exps = local_exps + local_result

    if trav.from_sep_close_bigger_starts is not None:
        direct = wrangler.eval_direct(
            actx, trav.target_boxes, trav.from_sep_close_bigger_starts,
            trav.from_sep_close_bigger_lists, src_weight_vecs)
        potentials = [a + b for a, b in zip(potentials, direct)]

    return _finish(actx, wrangler, trav, potentials, local_exps)


def _finish(actx, wrangler, trav, potentials, local_exps):
    local_exps = wrangler.refine_locals(
        actx, trav.level_start_target_or_target_parent_box_nrs,
        trav.target_or_target_parent_boxes, local_exps)

    local_result = wrangler.eval_locals(
        actx, trav.level_start_target_box_nrs, trav.target_boxes, local_exps)
    potentials = [a + b for a, b in zip(potentials, local_result)]

    result = wrangler.reorder_potentials(potentials)
    return wrangler.finalize_potentials(actx, result)


def _drive_concurrent(actx, wrangler, trav, src_weight_vecs, crit, side):
    """The chain on ``crit``; List 4, List 3 and List 1 on ``side`` in that
    order. The chain waits for List 4 alone before L2L (its locals join the
    List-2 locals there), so List 1 -- the longest independent stage -- runs
    beside the chain's latency-bound L2L levels and L2P; the potentials of
    Lists 1 and 3 join after L2P."""
    import torch
    main = torch.cuda.current_stream(crit.device)
    getattr(wrangler, "_geom", None)             # shared device geometry, made on this stream
    crit.wait_stream(main)                       # strengths reordered
    side.wait_stream(main)
    for t in src_weight_vecs:
        t.record_stream(crit)
        t.record_stream(side)
    with torch.cuda.stream(crit):
        mpole_exps = wrangler.form_multipoles(
            actx, trav.level_start_source_box_nrs, trav.source_boxes, src_weight_vecs)
        mpole_exps = wrangler.coarsen_multipoles(
            actx, trav.level_start_source_parent_box_nrs, trav.source_parent_boxes,
            mpole_exps)
        wrangler.communicate_mpoles(actx, mpole_exps)
    with torch.cuda.stream(side):
        local_result = wrangler.form_locals(
            actx, trav.level_start_target_or_target_parent_box_nrs,
            trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
            trav.from_sep_bigger_lists, src_weight_vecs)
        list4_done = torch.cuda.Event()
        list4_done.record(side)
        side.wait_stream(crit)                   # multipoles finished
        mpole_result = wrangler.eval_multipoles(
            actx, trav.target_boxes_sep_smaller_by_source_level,
            trav.from_sep_smaller_by_level, mpole_exps)
        potentials = wrangler.eval_direct(
            actx, trav.target_boxes, trav.neighbor_source_boxes_starts,
            trav.neighbor_source_boxes_lists, src_weight_vecs)
        potentials = [a + b for a, b in zip(potentials, mpole_result)]
    mpole_exps.record_stream(side)
    with torch.cuda.stream(crit):
        local_exps = wrangler.multipole_to_local(
            actx, trav.level_start_target_or_target_parent_box_nrs,
            trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
            trav.from_sep_siblings_lists, mpole_exps)
        crit.wait_event(list4_done)
        local_result.record_stream(crit)
        local_exps = local_exps + local_result
        local_exps = wrangler.refine_locals(
            actx, trav.level_start_target_or_target_parent_box_nrs,
            trav.target_or_target_parent_boxes, local_exps)
        local_pot = wrangler.eval_locals(
            actx, trav.level_start_target_box_nrs, trav.target_boxes, local_exps)
        crit.wait_stream(side)                   # Lists 1 and 3 finished
        for t in potentials:
            t.record_stream(crit)
        for starts, lists in ((trav.from_sep_close_smaller_starts,
                               trav.from_sep_close_smaller_lists),
                              (trav.from_sep_close_bigger_starts,
                               trav.from_sep_close_bigger_lists)):
            if starts is not None:
                direct = wrangler.eval_direct(actx, trav.target_boxes, starts, lists,
                                              src_weight_vecs)
                potentials = [a + b for a, b in zip(potentials, direct)]
        potentials = [a + b for a, b in zip(potentials, local_pot)]
        result = wrangler.finalize_potentials(actx, wrangler.reorder_potentials(potentials))
    main.wait_stream(crit)
    for t in result:
        t.record_stream(main)
    return result
