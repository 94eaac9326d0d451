"""Benchmark: 3D Laplace FMM evaluation throughput on one B200 (or N replicas).

Headline workload (one step = one full FMM evaluation, ``drive_fmm``):
1,000,000 points that are both sources and targets (exclude_self), 50% on
the unit sphere surface and 50% Plummer (scale 0.1), strengths N(0, 1),
expansion order 10, max_particles_in_box 96. Synthetic, seeded inputs; the
tree, interaction lists and M2L tables are built once before timing
(reported separately). ``value`` is Mpts/s of the mixed-precision form with
inputs resident in HBM; the FP64 form is timed on the same tree for the
ratio; the accuracy of both is the relative L2 error on 4,096 sampled
targets against an FP64 direct sum. Order 10 cannot reach relL2 <= 1e-6 on
this workload (the FP64 form gives 3.4e-6), so the line also carries the
same workload at the lowest order that does (``accuracy_target``: mixed and
FP64 on one tree). ``e2e`` runs the public API with host buffers (H2D of
the strengths, D2H of the potentials inside the timed region).

A default run prints that one JSON line and nothing else on stdout, as soon
as it is measured; progress goes to stderr with timestamps, and a section
that runs longer than ``--stall-dump-s`` dumps every thread's Python stack to
stderr. ``--extras`` adds the other workloads (adjoint, 512-problem batch,
Helmholtz, 20k uniform case, interaction matrices, QBX layer potentials),
each as a JSON line of
its own after the headline, within ``--budget-s``.

The CPU baseline is the oracle (C + OpenMP, sumpy's algorithm restated) on
the headline workload itself, one evaluation, run in a child process that
never imports torch and is killed if it overruns ``--cpu-timeout-s``.

``--impl reference`` times that oracle on the headline workload (same tree,
order and leaf size; W warm-up and K timed evaluations) and prints the same
metric; when K + W full evaluations would not fit ``--ref-budget-s`` it
times a sample of the workload instead and says so (``same_config``).

Multi-GPU (torchrun): each rank evaluates its own replica; no collective on
the data path (the problem does not shard in this build); value = points of
all ranks / max over ranks of the step time.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "3D Laplace FMM Mpts/s @ relL2<=1e-6 (mixed vs FP64 GPU); adjoint/forward ratio"
NPOINTS = 1_000_000
ORDER = 10
# max_particles_in_box of the 1M-point workload (the workload leaves it open): the fastest
# mixed form in a sweep over 32..192 on this GPU (32: 11.0 ms, 64: 10.1, 96: 9.6, 128: 10.0,
# 192: 13.7 ms; accuracy against the direct sum 3.5e-6 for all). The FP64 form is timed on
# the same tree (like for like) and, with --extras, on its own fastest tree.
MAX_PARTICLES = 96
FP64_MAX_PARTICLES = 128
HELMHOLTZ_MAX_PARTICLES = 64   # same sweep for the Helmholtz workload: 32: 46 ms, 64: 21 ms
BATCH_MAX_PARTICLES = 32       # the batched workload's own setting
ADJOINT_MAX_PARTICLES = 32
# the order that meets relL2 <= 1e-6 on the headline workload (p = 11: 1.7e-6,
# p = 12: 1.02e-6, p = 13: 9.6e-7 in the mixed form), on its own leaf-128 tree
ACCURACY_ORDER = 13
ACCURACY_MAX_PARTICLES = 128
NSAMPLE = 4096

_T0 = time.perf_counter()
_STALL_DUMP_S = 240.0


def progress(msg):
    """Timestamped progress on stderr; re-arms the stall dump (a section that
    runs past the limit prints every thread's Python stack to stderr)."""
    print(f"[bench {time.perf_counter() - _T0:8.1f} s] {msg}", file=sys.stderr, flush=True)
    if _STALL_DUMP_S > 0:
        faulthandler.dump_traceback_later(_STALL_DUMP_S, repeat=True, file=sys.stderr)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--npoints", type=int, default=NPOINTS)
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-timeout-s", type=float, default=240.0,
                    help="kill the CPU-baseline child process after this long")
    ap.add_argument("--ref-budget-s", type=float, default=900.0,
                    help="--impl reference: time budget of the W + K evaluations")
    ap.add_argument("--budget-s", type=float, default=1500.0,
                    help="wall-clock budget: sections that would start later are skipped "
                         "and listed under 'skipped'")
    ap.add_argument("--stall-dump-s", type=float, default=240.0,
                    help="dump all Python stacks to stderr when one section runs this long "
                         "(0: off)")
    ap.add_argument("--no-fp64", action="store_true", help="skip timing the FP64 form")
    ap.add_argument("--no-accuracy-target", action="store_true",
                    help="skip the accuracy-target order (p = 13) of the headline workload")
    ap.add_argument("--extras", action="store_true",
                    help="after the headline, run the other workloads (one JSON line each)")
    ap.add_argument("--only", choices=["mixed", "fp64", "batch", "helmholtz", "uniform",
                                       "matrix", "adjoint", "qbx", "m2l_mixed", "m2l_fp64"],
                    help="run one workload alone (--steps/--warmup apply) and print its result; "
                         "for profiling")
    ap.add_argument("--eager", action="store_true",
                    help="with --only: launch kernel by kernel instead of replaying a CUDA graph")
    ap.add_argument("--helmholtz-npoints", type=int, default=500_000)
    ap.add_argument("--helmholtz-precision", choices=["mixed", "fp64", "both"], default="both")
    return ap.parse_args()


def workload(npoints, seed=2024):
    from tests._pointsets import sphere_plummer
    pts = sphere_plummer(npoints, seed)
    q = np.random.default_rng(44).standard_normal(npoints)
    return pts, q


# {{{ reference arm / CPU baseline (oracle)

def run_reference(args):
    """The oracle (FP64 C + OpenMP restatement of sumpy's wrangler stages,
    ``sumpy/fmm.py:609-1083``) on the headline workload: the same points,
    tree (leaf size), order and exclude_self as the GPU arm. The first
    warm-up evaluation sizes the run: if W + K full evaluations would exceed
    ``--ref-budget-s``, each step becomes a sample of the workload (fewer
    points, same distribution) sized to fit, and the line says so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from sumpy_b200.tree import build_all
    progress(f"reference: workload {args.npoints} points, p = {args.order}")
    pts, q = workload(args.npoints)
    tree, trav, tcls = build_all(pts, None, MAX_PARTICLES)
    n = args.npoints

    def step():
        t0 = time.perf_counter()
        O.run_fmm(tree, trav, tcls, args.order, q, exclude_self=True)
        return time.perf_counter() - t0

    times = []
    progress("reference: first evaluation (sizes the run)")
    t1 = step()
    if args.warmup == 0:
        times.append(t1)          # the first timed step also sized the run
    left = max(args.warmup - 1, 0) + args.steps - len(times)
    same = left * t1 <= args.ref_budget_s
    if not same:
        # a sample of the same distribution whose W + K evaluations fit the budget
        n = max(20_000, int(args.npoints * args.ref_budget_s /
                            (max(args.warmup + args.steps, 1) * t1)))
        n = min(n, args.npoints)
        progress(f"reference: {left} full evaluations would take {left * t1:.0f} s; "
                 f"timing a {n}-point sample instead")
        pts, q = workload(n)
        tree, trav, tcls = build_all(pts, None, MAX_PARTICLES)
        times = []
        for _ in range(args.warmup):
            step()
    else:
        for _ in range(max(args.warmup - 1, 0)):
            step()
    progress(f"reference: {args.steps} timed evaluations ({t1:.1f} s each)")
    while len(times) < args.steps:
        times.append(step())
    tot = sum(times)
    value = n * args.steps / tot / 1e6
    cores = O.num_threads()
    sample = (f"the headline workload itself ({n} points, p={args.order}, leaf "
              f"{MAX_PARTICLES}), FP64 C/OpenMP oracle (sumpy's algorithm restated), "
              f"{cores} threads, {tot / args.steps:.1f} s per evaluation"
              if same else
              f"{n}-point sample of the headline distribution, p={args.order}, leaf "
              f"{MAX_PARTICLES}: {args.warmup + args.steps} evaluations of all "
              f"{args.npoints} points at "
              f"{t1:.1f} s would exceed {args.ref_budget_s:.0f} s; FP64 C/OpenMP oracle, "
              f"{cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"laplace3d_fmm_sphere_plummer_n{args.npoints}_p{args.order}",
                   "npoints": args.npoints, "order": args.order,
                   "max_particles_in_box": MAX_PARTICLES, "exclude_self": True,
                   "same_config": same, "points_per_step": n},
        "cpu_baseline": {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    faulthandler.cancel_dump_traceback_later()
    print(json.dumps(line), flush=True)


def cpu_baseline_child(args):
    """One oracle evaluation of the headline workload, timed in a child
    process (``--impl reference --steps 1 --warmup 0``) that never imports
    torch; None (with the reason) when it fails or overruns."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE")}
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
           "--warmup", "0", "--npoints", str(args.npoints), "--order", str(args.order),
           "--ref-budget-s", str(0.5 * args.cpu_timeout_s),
           "--stall-dump-s", str(args.stall_dump_s)]
    try:
        res = subprocess.run(cmd, capture_output=True, text=True, env=env,
                             timeout=args.cpu_timeout_s)
    except subprocess.TimeoutExpired as e:
        err = (e.stderr or b"")
        err = err.decode(errors="replace") if isinstance(err, bytes) else err
        sys.stderr.write(err[-4000:])
        return None, f"oracle child process overran {args.cpu_timeout_s:.0f} s (killed)"
    sys.stderr.write(res.stderr[-4000:])
    if res.returncode != 0:
        return None, f"oracle child process exited {res.returncode}"
    try:
        ref = json.loads(res.stdout.strip().splitlines()[-1])
    except (ValueError, IndexError):
        return None, "oracle child process printed no result line"
    cb = dict(ref["cpu_baseline"])
    cb["same_config"] = ref["config"]["same_config"]
    return cb, None

# }}}
class ClockSampler:
    """SM clock and clock-event reasons sampled DURING a timed region by a
    daemon thread: NVML polled every 5 ms (read-only queries), so that even a
    region of a few tens of milliseconds gets samples; nvidia-smi at its
    100 ms floor when NVML is unavailable. Every NVML call, its
    initialisation included, runs in that thread: the timed thread never
    waits on NVML, and leaving the region waits at most a few seconds for
    the sampler to stop (a sampler that did not answer leaves no samples,
    and the summary says so)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index, period_s=0.005):
        import threading
        self.gpu = gpu_index
        self.period = period_s
        self.proc = None
        self.thread = None
        self.samples = []
        self.max_mhz = None
        self.source = None
        self.uuid = None
        self._stop = threading.Event()

    def _nvml(self):
        import pynvml as nv
        nv.nvmlInit()
        h = None
        if self.uuid:
            for cand in (self.uuid, "GPU-" + self.uuid):
                try:
                    h = nv.nvmlDeviceGetHandleByUUID(cand)
                    break
                except Exception:  # noqa: BLE001
                    h = None
        if h is None:
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        bits = [("hw_slowdown", nv.nvmlClocksEventReasonHwSlowdown),
                ("hw_thermal_slowdown", nv.nvmlClocksEventReasonHwThermalSlowdown),
                ("sw_thermal_slowdown", nv.nvmlClocksEventReasonSwThermalSlowdown),
                ("sw_power_cap", nv.nvmlClocksEventReasonSwPowerCap)]
        self.source = "nvml"
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), [n for n, b in bits if rs & b]))
            except Exception:  # noqa: BLE001 (a failed read is skipped)
                pass
            self._stop.wait(self.period)

    def _smi(self):
        self.source = "nvidia-smi"
        self.proc = subprocess.Popen(
            ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
             "--format=csv,noheader,nounits", "-lms", "100"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        for r in self.proc.stdout:
            if self._stop.is_set():
                break
            r = [x.strip() for x in r.split(",")]
            if len(r) < 9:
                continue
            try:
                sm = float(r[1])
                self.max_mhz = float(r[2])
            except ValueError:
                continue
            self.samples.append(
                (sm, [nm for nm, v in zip(self.NAMES, r[5:9]) if v.lower() == "active"]))

    def _run(self):
        try:
            self._nvml()
            return
        except Exception:  # noqa: BLE001 (no NVML: fall back to nvidia-smi)
            pass
        try:
            self._smi()
        except Exception:  # noqa: BLE001 (no sampler at all: no samples)
            pass

    def __enter__(self):
        import threading
        try:
            import torch
            self.uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
        except Exception:  # noqa: BLE001
            self.uuid = None
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=3)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.thread.join(timeout=3)

    def summary(self):
        samples = list(self.samples)
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0,
                    "source": self.source, "note": "the clock sampler took no sample"}
        reasons = sorted({n for _, rs in samples for n in rs})
        return {"sm_mhz": float(np.median([s for s, _ in samples])),
                "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(samples), "source": self.source}


class Budget:
    """Wall-clock budget of the whole run: ``ok(name, need_s)`` says whether
    a section expected to take ``need_s`` seconds may still start, and
    records the ones that may not."""

    def __init__(self, seconds):
        self.seconds = seconds
        self.skipped = []

    def elapsed(self):
        return time.perf_counter() - _T0

    def ok(self, name, need_s=0.0):
        if self.elapsed() + need_s > self.seconds:
            self.skipped.append(name)
            progress(f"skip {name}: {self.elapsed():.0f} s used of {self.seconds:.0f} s")
            return False
        return True


def main():
    global _STALL_DUMP_S
    args = parse()
    _STALL_DUMP_S = args.stall_dump_s
    faulthandler.enable(file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
        return
    budget = Budget(args.budget_s)
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))

    # CPU baseline first, in a child process without torch, before this
    # process loads CUDA or competes for the host cores
    cpu_line, cpu_why = None, "not run (--no-cpu-baseline, --only or N > 1)"
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.only is None:
        progress("cpu baseline: oracle child process")
        cpu_line, cpu_why = cpu_baseline_child(args)
        progress(f"cpu baseline: {cpu_line['value']:.4f} Mpts/s" if cpu_line else
                 f"cpu baseline: none ({cpu_why})")

    progress("import torch")
    import torch

    from sumpy_b200.distributed import init as dist_init
    rank, world, local_rank = dist_init("nccl", timeout_s=300)
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    from sumpy_b200 import _lib
    _lib.load_cuda_library()

    if args.only is not None:
        res = run_only(args, dev)
        if rank == 0:
            print(json.dumps({"only": args.only, "result": res}), flush=True)
        faulthandler.cancel_dump_traceback_later()
        return

    line = headline(args, dev, rank, world, local_rank, budget, cpu_line, cpu_why)
    if rank == 0:
        print(json.dumps(line), flush=True)
    progress("headline printed")

    if args.extras and world == 1:
        for name, fn in (("fp64_own_best_tree", lambda: fp64_best_tree_bench(dev, args)),
                         ("batched", lambda: batched_bench(dev)),
                         ("helmholtz", lambda: helmholtz_bench(dev)),
                         ("uniform_p6", lambda: uniform_bench(dev)),
                         ("p2p_matrix", lambda: matrix_bench(dev)),
                         ("qbx", lambda: qbx_bench(dev))):
            if not budget.ok(name, 30.0):
                continue
            progress(f"extra: {name}")
            import gc
            gc.collect()
            torch.cuda.empty_cache()
            res = fn()
            print(json.dumps({"extra": name, "result": res}), flush=True)
        if budget.skipped:
            print(json.dumps({"extra": "skipped", "result": budget.skipped}), flush=True)
    faulthandler.cancel_dump_traceback_later()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def laplace_setup(dev, npoints, max_particles):
    """Points, strengths, tree and the tree-independent data of the headline
    workload. The tree is built on the GPU (``sumpy_tree_gpu_build``) from
    the points in device memory; the time covers the build and the host
    copies of its arrays."""
    import torch
    from sumpy_b200 import LaplaceKernel, SumpyTreeIndependentDataForWrangler
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    pts, q = workload(npoints)
    pts_dev = torch.as_tensor(pts, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tree, trav, tcls = build_all(pts_dev, None, max_particles)
    t_tree = time.perf_counter() - t0
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    return pts, q, tree, trav, tcls, ti, t_tree


def make_wrangler(ti, trav, tcls, order, precision, dev, graph=True):
    """An expansion wrangler of one order on every level; ``graph``: drive_fmm
    replays the evaluation from a CUDA graph (one host call per step)."""
    from sumpy_b200 import SumpyExpansionWrangler
    return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev, p=order: p,
                                  translation_classes_data=tcls, precision=precision,
                                  device=dev, cuda_graph=graph)


class StepTimer:
    """Per-step CUDA-event times on the current stream with an L2 flush (a
    256 MB write, outside the events) before every step; barrier +
    synchronize on both sides; the max over ranks of the mean step time."""

    def __init__(self, dev, world):
        import torch
        self.dev = dev
        self.world = world
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def _barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def __call__(self, fn, steps):
        import torch
        from sumpy_b200.distributed import max_over_ranks
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        self._barrier()
        for i in range(steps):
            self.flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        self._barrier()
        ms = [a.elapsed_time(b) for a, b in evs]
        return max_over_ranks(sum(ms), device=self.dev) / steps, ms


def headline(args, dev, rank, world, local_rank, budget, cpu_line, cpu_why):
    """The headline line: mixed form (graph replay, timed, with clocks and
    launch count), its eager launches, e2e with host buffers, the FP64 form
    on the same tree, accuracy on sampled targets, the accuracy-target
    order, the adjoint through the autograd API, stage times and the
    roofline of the dominant kernel."""
    import torch
    from sumpy_b200 import P2P, LaplaceKernel, _capi, drive_fmm

    progress("headline: workload and tree")
    pts, q, tree, trav, tcls, ti, t_tree = laplace_setup(dev, args.npoints, MAX_PARTICLES)
    t0 = time.perf_counter()
    from sumpy_b200.tree import build_all
    build_all(pts, None, MAX_PARTICLES)
    t_tree_host = time.perf_counter() - t0
    timer = StepTimer(dev, world)
    q_dev = torch.as_tensor(q, device=dev)

    progress("headline: mixed form set-up (plans, tables, graph capture)")
    t0 = time.perf_counter()
    w_mx = make_wrangler(ti, trav, tcls, args.order, "mixed", dev)
    drive_fmm(None, w_mx, [q_dev])
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0

    progress("headline: mixed form, kernel-by-kernel launches")
    w_mx.cuda_graph = False
    for _ in range(max(1, args.warmup)):
        drive_fmm(None, w_mx, [q_dev])
    ms_eager, _ = timer(lambda: drive_fmm(None, w_mx, [q_dev]), args.steps)
    w_mx.cuda_graph = True

    progress("headline: mixed form, graph replay (the timed value)")
    # the sampler starts with the warm-up steps, so that it samples from the
    # first timed step on
    with ClockSampler(local_rank) as clk:
        for _ in range(args.warmup):
            drive_fmm(None, w_mx, [q_dev])
        _capi.launch_counter.reset()
        ms_mx, _ = timer(lambda: drive_fmm(None, w_mx, [q_dev]), args.steps)
        launches = _capi.launch_counter.value
    clocks = clk.summary()
    w_mx.check_status()

    progress("headline: e2e through the public API with pinned host buffers")
    q_host = torch.as_tensor(q).pin_memory()
    pot_host = torch.empty(args.npoints, dtype=torch.float64).pin_memory()

    def e2e_step():
        # strengths copied from pinned host memory into the graph's input,
        # potentials copied back to pinned host memory, both inside the events
        (pot,) = drive_fmm(None, w_mx, [q_host])
        pot_host.copy_(pot, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    ms_e2e, _ = timer(e2e_step, args.steps)

    ms_64, w_64 = None, None
    if not args.no_fp64 and (world > 1 or budget.ok("fp64", 20.0)):
        progress("headline: FP64 form on the same tree")
        w_64 = make_wrangler(ti, trav, tcls, args.order, "fp64", dev)
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w_64, [q_dev])
        ms_64, _ = timer(lambda: drive_fmm(None, w_64, [q_dev]), args.steps)
        w_64.check_status()

    progress("headline: accuracy on sampled targets against the FP64 direct sum")
    knl = LaplaceKernel(3)
    rng = np.random.default_rng(99)
    sample = rng.choice(args.npoints, size=min(NSAMPLE, args.npoints), replace=False)
    (ref,) = P2P([knl], exclude_self=True)(None, pts[:, sample], pts, (q,),
                                           target_to_source=sample, device=dev)
    ref = ref.cpu().numpy()

    def rel(w):
        p = drive_fmm(None, w, [q_dev])[0].cpu().numpy()
        return float(np.linalg.norm(p[sample] - ref) / np.linalg.norm(ref))

    err_mx = rel(w_mx)
    err_64 = rel(w_64) if w_64 is not None else None
    del w_64
    torch.cuda.empty_cache()

    # the metric's accuracy condition on the same workload: the lowest order
    # that reaches it, mixed and FP64 forms on one tree
    at = None
    if (not args.no_accuracy_target and args.npoints == NPOINTS and args.order == ORDER
            and world == 1 and budget.ok("accuracy_target", 60.0)):
        at = accuracy_target(args, dev, pts, q_dev, ti, timer, rel)

    adj = None
    if world == 1 and budget.ok("adjoint", 60.0):
        progress("headline: adjoint through the autograd API (200k -> 50k, p = 8)")
        adj = adjoint_api_bench(dev, steps=max(3, min(args.steps, 10)))

    progress("headline: stage times and roofline")
    pipes = pipe_peaks_measured(dev)
    stage_ms, roof, roof_m2l = stage_breakdown(w_mx, trav, q_dev, dev, pipe_peaks=pipes)

    value = world * args.npoints / (ms_mx * 1e-3) / 1e6
    return {
        "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mx,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/3xf16 (row-scaled) with f64 offsets and sums", "data": "synthetic",
        "config": {
            "workload": f"laplace3d_fmm_sphere_plummer_n{args.npoints}_p{args.order}",
            "npoints": args.npoints, "order": args.order,
            "max_particles_in_box": MAX_PARTICLES, "exclude_self": True,
            "precision": "mixed (FP32 near field, M2P, P2L with FP64 offsets and sums; "
                         "tensor-core M2L with row-scaled split-f16 operands (3 products, "
                         "FP32 sums per class group, FP64 across groups); FP64 elsewhere)",
            "accuracy_target": (f"relL2 <= 1e-6 reached at p = {at['order']}, leaf "
                                f"{ACCURACY_MAX_PARTICLES} (accuracy_target)") if at else None,
            "l2": "flushed between steps (256 MB write outside the timed events)",
            "parallelism": f"replicas x{world}",
            "launch": "drive_fmm replaying a CUDA graph of the whole evaluation "
                      "(wrangler cuda_graph=True); kernel-by-kernel timing beside it",
            "tree_build_s": round(t_tree, 4),
            "tree_build": "GPU (sumpy_tree_gpu_build) incl. host copies of the arrays; "
                          f"the host builder takes {t_tree_host:.3f} s for the same tree",
            "setup_s": round(t_setup, 3),
        },
        "eager": {"ms_per_step": ms_eager,
                  "value": world * args.npoints / (ms_eager * 1e-3) / 1e6},
        "accuracy": {"relL2_mixed": err_mx, "relL2_fp64": err_64,
                     "targets_sampled": len(sample),
                     "reference": "FP64 direct sum (GPU kernel sumpy_p2p_direct_f64)"},
        "fp64": {"value": (world * args.npoints / (ms_64 * 1e-3) / 1e6) if ms_64 else None,
                 "ms_per_step": ms_64},
        "mixed_over_fp64": (ms_64 / ms_mx) if ms_64 else None,
        "accuracy_target": at,
        "mixed_over_fp64_at_accuracy_target": at.get("mixed_over_fp64") if at else None,
        "adjoint_forward_ratio": adj["ratio"] if adj else None,
        "adjoint": adj,
        "stage_ms": stage_ms,
        "roofline": roof,
        "roofline_m2l": roof_m2l,
        "measured_pipe_peaks": pipes,
        "cpu_baseline": cpu_line if cpu_line else {"value": None, "why": cpu_why},
        "e2e": {"value": world * args.npoints / (ms_e2e * 1e-3) / 1e6, "unit": "Mpts/s",
                "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": 8 * args.npoints, "d2h_bytes_per_step": 8 * args.npoints},
        "gpu_launches": launches,
        "clocks": clocks,
        "skipped": list(budget.skipped),
    }


def accuracy_target(args, dev, pts, q_dev, ti, timer, rel):
    """The headline workload at the lowest order that meets relL2 <= 1e-6
    (ACCURACY_ORDER, one more if it does not), mixed and FP64 forms on one
    leaf-128 tree, timed like the headline."""
    import torch
    from sumpy_b200 import drive_fmm
    from sumpy_b200.tree import build_all
    progress(f"headline: accuracy target (p = {ACCURACY_ORDER}, leaf {ACCURACY_MAX_PARTICLES})")
    tree_a, trav_a, tcls_a = build_all(pts, None, ACCURACY_MAX_PARTICLES)
    out = None
    for p_hi in (ACCURACY_ORDER, ACCURACY_ORDER + 1):
        w_p = make_wrangler(ti, trav_a, tcls_a, p_hi, "mixed", dev)
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w_p, [q_dev])
        ms_p, _ = timer(lambda: drive_fmm(None, w_p, [q_dev]), args.steps)
        e_p = rel(w_p)
        w_p.check_status()
        out = {"order": p_hi, "max_particles_in_box": ACCURACY_MAX_PARTICLES,
               "ms_per_step": ms_p, "value": args.npoints / (ms_p * 1e-3) / 1e6,
               "relL2_mixed": e_p, "meets_1e-6": e_p <= 1e-6}
        del w_p
        if e_p <= 1e-6:
            break
    if not args.no_fp64:
        progress(f"headline: accuracy target, FP64 form at p = {out['order']}")
        w_f = make_wrangler(ti, trav_a, tcls_a, out["order"], "fp64", dev)
        for _ in range(max(1, args.warmup)):
            drive_fmm(None, w_f, [q_dev])
        ms_f, _ = timer(lambda: drive_fmm(None, w_f, [q_dev]), args.steps)
        e_f = rel(w_f)
        w_f.check_status()
        out.update({"fp64_ms_per_step": ms_f,
                    "fp64_value": args.npoints / (ms_f * 1e-3) / 1e6, "relL2_fp64": e_f,
                    "mixed_over_fp64": ms_f / out["ms_per_step"]})
        del w_f
    torch.cuda.empty_cache()
    return out


def run_only(args, dev):
    """One workload alone (profiling): --only mixed|fp64 run the headline
    workload in that form (graph replay, or --eager)."""
    import torch
    from sumpy_b200 import drive_fmm
    if args.only == "batch":
        return batched_bench(dev, steps=args.steps, warmup=args.warmup)
    if args.only == "matrix":
        return matrix_bench(dev, steps=args.steps, warmup=args.warmup)
    if args.only == "uniform":
        return uniform_bench(dev, steps=args.steps, warmup=args.warmup, cpu=False)
    if args.only == "adjoint":
        return adjoint_api_bench(dev, steps=args.steps, warmup=args.warmup)
    if args.only == "qbx":
        return qbx_bench(dev, steps=args.steps, warmup=args.warmup)
    if args.only == "helmholtz":
        precs = (("mixed", "fp64") if args.helmholtz_precision == "both"
                 else (args.helmholtz_precision,))
        return helmholtz_bench(dev, steps=args.steps, warmup=args.warmup,
                               npoints=args.helmholtz_npoints, precisions=precs)
    if args.only in ("m2l_mixed", "m2l_fp64"):
        return m2l_alone(args, dev, args.only[4:])
    pts, q, tree, trav, tcls, ti, t_tree = laplace_setup(dev, args.npoints, MAX_PARTICLES)
    w = make_wrangler(ti, trav, tcls, args.order, args.only, dev, graph=not args.eager)
    q_dev = torch.as_tensor(q, device=dev)
    for _ in range(max(1, args.warmup)):
        drive_fmm(None, w, [q_dev])
    ms, _ = StepTimer(dev, 1)(lambda: drive_fmm(None, w, [q_dev]), args.steps)
    w.check_status()
    return {"ms_per_step": ms, "Mpts_s": args.npoints / (ms * 1e-3) / 1e6}


def m2l_alone(args, dev, precision):
    """The headline workload's M2L (all levels) alone, for profiling: one
    full FMM for the multipoles, W untimed and K timed ``multipole_to_local``
    calls (CUDA events), the last of them inside the NVTX range "m2l"."""
    import torch
    from sumpy_b200 import drive_fmm
    pts, q, tree, trav, tcls, ti, _ = laplace_setup(dev, args.npoints, MAX_PARTICLES)
    w = make_wrangler(ti, trav, tcls, args.order, precision, dev, graph=False)
    qd = torch.as_tensor(q, device=dev)
    drive_fmm(None, w, [qd])
    qs = w.reorder_sources(qd)
    mp = w.coarsen_multipoles(
        None, trav.level_start_source_parent_box_nrs, trav.source_parent_boxes,
        w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs]))
    m2l_args = (None, trav.level_start_target_or_target_parent_box_nrs,
                trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
                trav.from_sep_siblings_lists, mp)
    for _ in range(max(1, args.warmup)):
        w.multipole_to_local(*m2l_args)
    torch.cuda.synchronize()
    times = []
    for i in range(max(1, args.steps)):
        last = i == max(1, args.steps) - 1
        if last:
            torch.cuda.nvtx.range_push("m2l")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        w.multipole_to_local(*m2l_args)
        e1.record()
        if last:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    w.check_status()
    return {"precision": precision, "m2l_ms": sorted(times)[len(times) // 2],
            "entries": int(len(trav.from_sep_siblings_lists))}


def fp64_best_tree_bench(dev, args):
    """The FP64 form on its own fastest tree (larger leaves favour its M2L)."""
    import torch
    from sumpy_b200 import drive_fmm
    pts, q, tree, trav, tcls, ti, _ = laplace_setup(dev, args.npoints, FP64_MAX_PARTICLES)
    w = make_wrangler(ti, trav, tcls, args.order, "fp64", dev)
    q_dev = torch.as_tensor(q, device=dev)
    for _ in range(max(1, args.warmup)):
        drive_fmm(None, w, [q_dev])
    ms, _ = StepTimer(dev, 1)(lambda: drive_fmm(None, w, [q_dev]), args.steps)
    return {"max_particles_in_box": FP64_MAX_PARTICLES, "ms_per_step": ms,
            "value": args.npoints / (ms * 1e-3) / 1e6}


def adjoint_problem(ns=200_000, nt=50_000, seed=7):
    """The differentiable-potential workload: ns sources on the unit sphere
    perturbed radially by 0.05*N(0,1), nt targets uniform in the shell
    2 <= r <= 3, strengths N(0,1); also the unperturbed sphere points."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((3, ns))
    u = g / np.linalg.norm(g, axis=0)
    src = (1 + 0.05 * rng.standard_normal(ns)) * u
    d = rng.standard_normal((3, nt))
    d /= np.linalg.norm(d, axis=0)
    tgt = np.cbrt(8 + 19 * rng.random(nt)) * d
    q = rng.standard_normal(ns)
    return src, tgt, q, u


def adjoint_api_bench(dev, steps=5, warmup=3, ns=200_000, nt=50_000, order=8, fd_check=True):
    """Backward/forward time of the differentiable potential through the API
    users call, :class:`sumpy_b200.autograd.LaplaceFMM` (mixed, p = 8): 200k
    perturbed sphere sources, 50k shell targets, loss 0.5*|phi - phi_ref|^2
    with phi_ref the FP64 direct sum at the unperturbed positions. A step is
    ``phi = fmm(q, x_s, x_t)`` and the loss (forward) then ``loss.backward()``
    (strength and source-position gradients); strengths and source positions
    are fresh leaf tensors each step. The first call builds the geometry;
    later calls find every point inside its box and reuse it. CUDA events
    around each part; gradients checked against the FP64 direct-sum
    gradients."""
    import torch
    from sumpy_b200 import P2P, LaplaceKernel
    from sumpy_b200.autograd import LaplaceFMM
    src, tgt, q, u = adjoint_problem(ns, nt)
    knl = [LaplaceKernel(3)]
    (phi_ref,) = P2P(knl)(None, tgt, u, (q,), device=dev)
    fmm = LaplaceFMM(order=order, max_particles_in_box=ADJOINT_MAX_PARTICLES,
                     precision="mixed", device=dev)
    q0 = torch.as_tensor(q, device=dev)
    s0 = torch.as_tensor(src, device=dev)
    t0 = torch.as_tensor(tgt, device=dev)

    def forward():
        qv = q0.clone().requires_grad_(True)
        sv = s0.clone().requires_grad_(True)
        phi = fmm(qv, sv, t0)
        loss = 0.5 * ((phi - phi_ref) ** 2).sum()
        return loss, qv, sv, phi

    tb = time.perf_counter()
    loss, qv, sv, phi = forward()
    loss.backward()
    torch.cuda.synchronize()
    t_first = time.perf_counter() - tb
    for _ in range(warmup):
        loss, qv, sv, phi = forward()
        loss.backward()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    torch.cuda.synchronize()
    for e in evs:
        e[0].record()
        loss, qv, sv, phi = forward()
        e[1].record()
        loss.backward()
        e[2].record()
    torch.cuda.synchronize()
    t_f = sum(e[0].elapsed_time(e[1]) for e in evs) / steps
    t_b = sum(e[1].elapsed_time(e[2]) for e in evs) / steps
    gdn = (phi - phi_ref).detach().cpu().numpy()
    psi = P2P(knl, gradient=True)(None, src, tgt, (gdn,), device=dev)
    gq_ref = psi[0]
    gsrc_ref = q0 * torch.stack(psi[1:4])
    rel = lambda a, b: float((a - b).norm() / b.norm())
    fd = adjoint_fd_check(dev, fmm, q0, s0, t0, phi_ref, order) if fd_check else None
    return {"forward_ms": t_f, "backward_ms": t_b, "ratio": t_b / t_f,
            "fd_check": fd,
            "api": "sumpy_b200.autograd.LaplaceFMM (torch.autograd.Function), "
                   "forward = fmm + loss, backward = loss.backward()",
            "first_call_s": round(t_first, 3),
            "geometry_builds": fmm.geometry_builds, "geometry_reuses": fmm.geometry_reuses,
            "grad_strength_relL2_vs_direct": rel(qv.grad, gq_ref),
            "grad_source_pos_relL2_vs_direct": rel(sv.grad, gsrc_ref),
            "workload": f"sphere(perturbed) {ns} sources -> shell {nt} targets, p={order}, "
                        f"mixed, leaf {ADJOINT_MAX_PARTICLES}"}


def adjoint_fd_check(dev, fmx, q0, s0, t0, phi_ref, order, h=1e-4, ncoord=32, seed=11):
    """Central differences (h = 1e-4, FP64 forward on the same boxes) of the
    loss on ``ncoord`` random strengths and ``ncoord`` random source
    coordinates (points at least 2h inside their boxes, so the geometry is
    reused), against: the FP64 adjoint, the mixed adjoint applied to the
    FP64 residual (the backward's own precision), and the mixed end-to-end
    gradient (which also carries the mixed forward's error, amplified by the
    small residual). Relative L2 over each set of coordinates."""
    import torch
    from sumpy_b200.autograd import LaplaceFMM
    f64 = LaplaceFMM(order=order, max_particles_in_box=ADJOINT_MAX_PARTICLES,
                     precision="fp64", device=dev)

    def grads(fmm, seed_residual=None):
        qv = q0.clone().requires_grad_(True)
        sv = s0.clone().requires_grad_(True)
        phi = fmm(qv, sv, t0)
        if seed_residual is None:
            (0.5 * ((phi - phi_ref) ** 2).sum()).backward()
        else:
            phi.backward(seed_residual)
        return qv.grad, sv.grad

    g64 = grads(f64)
    gmx = grads(fmx)
    r64 = (f64(q0, s0, t0) - phi_ref).detach()
    gmb = grads(fmx, r64)

    def loss(qq, ss):
        return 0.5 * float(((f64(qq, ss, t0) - phi_ref) ** 2).sum())

    geo = f64._cache.geo
    lo, hi = geo.src_lo.cpu().numpy(), geo.src_hi.cpu().numpy()
    inv = np.empty(len(q0), dtype=np.int64)
    inv[geo.src_perm.cpu().numpy()] = np.arange(len(q0))
    xs = geo.src_sorted.cpu().numpy()
    rng = np.random.default_rng(seed)
    iq = rng.choice(len(q0), ncoord, replace=False)
    coords = []
    while len(coords) < ncoord:
        i, d = int(rng.integers(len(q0))), int(rng.integers(3))
        k = inv[i]
        if lo[d, k] < xs[d, k] - 2 * h and xs[d, k] + 2 * h < hi[d, k]:
            coords.append((d, i))
    fd_q, fd_x = [], []
    for i in iq:
        qp, qm = q0.clone(), q0.clone()
        qp[i] += h
        qm[i] -= h
        fd_q.append((loss(qp, s0) - loss(qm, s0)) / (2 * h))
    for d, i in coords:
        sp, sm = s0.clone(), s0.clone()
        sp[d, i] += h
        sm[d, i] -= h
        fd_x.append((loss(q0, sp) - loss(q0, sm)) / (2 * h))
    fd_q, fd_x = np.array(fd_q), np.array(fd_x)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    pq = lambda g: g[0][torch.as_tensor(iq, device=dev)].cpu().numpy()
    px = lambda g: np.array([g[1][d, i].item() for d, i in coords])
    return {"h": h, "coordinates": f"{ncoord} strengths + {ncoord} source coordinates",
            "geometry_builds_fp64": f64.geometry_builds,
            "fp64": {"strengths": rel(pq(g64), fd_q), "positions": rel(px(g64), fd_x)},
            "mixed_backward_on_fp64_residual": {"strengths": rel(pq(gmb), fd_q),
                                                "positions": rel(px(gmb), fd_x)},
            "mixed": {"strengths": rel(pq(gmx), fd_q), "positions": rel(px(gmx), fd_x)},
            "residual_over_phi": float((r64.norm() / (r64 + phi_ref).norm()).item())}


def batch_problems(nproblems=512):
    """The batched workload: problem i draws from seed 1000 + i its size
    N_i = floor(exp(U(ln 1000, ln 65536))), N_i points U[0,1]^3 (sources =
    targets) and N_i strengths N(0, 1)."""
    srcs, qs = [], []
    for i in range(nproblems):
        rng = np.random.default_rng(1000 + i)
        n = int(np.floor(np.exp(rng.uniform(np.log(1000), np.log(65536)))))
        srcs.append(rng.random((3, n)))
        qs.append(rng.standard_normal(n))
    return srcs, qs


def batched_bench(dev, steps=5, warmup=3, nproblems=512, order=8, nseq=16):
    """512 independent problems (p = 8, mixed, max 32 per box, exclude_self)
    as one forest: CUDA-graph replay and eager launches of the whole batch,
    against the same problems evaluated one drive_fmm at a time (the first
    ``nseq`` problems, rate extrapolated by points). Accuracy: relative L2
    error on 4 problems (512 sampled targets each) against the FP64 direct
    sum. L2 flushed between timed batches."""
    import torch
    from sumpy_b200 import (P2P, LaplaceKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200 import _capi
    from sumpy_b200.batch import BatchedLaplaceFMM
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    box = [[0.0, 1.0]] * 3
    srcs, qs = batch_problems(nproblems)
    ntot = sum(q.size for q in qs)
    t0 = time.perf_counter()
    b = BatchedLaplaceFMM(srcs, order=order, max_particles_in_box=BATCH_MAX_PARTICLES,
                          precision="mixed", bbox=box, device=dev, use_graph=True,
                          autotune=True)
    t_build = time.perf_counter() - t0
    w_dev = torch.as_tensor(np.concatenate(qs), device=dev)
    t0 = time.perf_counter()
    b.capture()
    t_capture = time.perf_counter() - t0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in evs) / steps

    ms_graph = timed(lambda: b.evaluate(w_dev))
    b.use_graph = False
    _capi.launch_counter.reset()
    b.evaluate(w_dev)
    launches = _capi.launch_counter.value
    ms_eager = timed(lambda: b.evaluate(w_dev))
    b.use_graph = True
    b.check_status()

    # one problem at a time (what a loop over sumpy FMMs does), first nseq problems
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    seq = []
    for i in range(nseq):
        _, trav, tcls = build_all(srcs[i], None, BATCH_MAX_PARTICLES, bbox=box)
        wr = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                                    translation_classes_data=tcls, precision="mixed",
                                    device=dev)
        seq.append((wr, torch.as_tensor(qs[i], device=dev)))
    nseq_pts = sum(q.numel() for _, q in seq)

    def run_seq():
        for wr, q in seq:
            drive_fmm(None, wr, [q])

    ms_seq = timed(run_seq)
    seq_rate = nseq_pts / (ms_seq * 1e-3) / 1e6

    # accuracy on 4 problems
    pots = b(w_dev)
    errs = []
    rng = np.random.default_rng(5)
    for i in (0, 1, nproblems // 2, nproblems - 1):
        n = qs[i].size
        smp = rng.choice(n, size=min(512, n), replace=False)
        (ref,) = P2P([knl], exclude_self=True)(None, srcs[i][:, smp], srcs[i], (qs[i],),
                                               target_to_source=smp, device=dev)
        ref = ref.cpu().numpy()
        got = pots[i].cpu().numpy()[smp]
        errs.append(float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
    return {
        "workload": f"{nproblems} problems U[0,1]^3, N_i=floor(exp(U(ln 1000, ln 65536))) "
                    f"(seed 1000+i), p={order}, mixed, exclude_self",
        "total_points": int(ntot), "nboxes": int(b.tree.nboxes),
        "graph": {"ms_per_batch": ms_graph, "Mpts_s": ntot / (ms_graph * 1e-3) / 1e6,
                  "problems_s": nproblems / (ms_graph * 1e-3)},
        "eager": {"ms_per_batch": ms_eager, "Mpts_s": ntot / (ms_eager * 1e-3) / 1e6,
                  "launches_per_batch": launches},
        "one_problem_at_a_time": {
            "Mpts_s": seq_rate, "problems_timed": nseq, "points_timed": int(nseq_pts),
            "ms_for_timed": ms_seq,
            "note": "drive_fmm per problem, warm, same kernels; whole-batch time "
                    "extrapolated by points"},
        "batch_over_one_at_a_time": (ntot / (ms_graph * 1e-3) / 1e6) / seq_rate,
        "schedule": b.schedule,
        "relL2_vs_direct": errs,
        "setup_s": round(t_build, 2),
        "forest_build_s": round(b.timings["forest_s"], 3),
        "autotune_s": round(b.timings.get("autotune_s", 0.0), 2),
        "setup_note": "setup_s = forest (GPU build and host copies of its arrays) + wrangler + "
                      "schedule autotuning (cached on disk after the first run); the work plans "
                      "are built by the first evaluation, inside capture_s",
        "capture_s": round(t_capture, 2),
    }


def matrix_bench(dev, steps=5, warmup=3, n=20_000, nsub=20_000_000):
    """Interaction matrices (P2PMatrixGenerator / P2PMatrixSubsetGenerator):
    the dense n x n Laplace matrix of n = 20k points U[0,1]^3 (3.2 GB of
    FP64 written; HBM-write bound: bytes = 8 per entry), the n/2 x n/2
    Helmholtz matrix (k = 10, 16 bytes per entry), and 20M random index
    pairs. CUDA-event time per call, inputs resident; roofline against the
    measured HBM copy bandwidth."""
    import torch
    from sumpy_b200 import (HelmholtzKernel, LaplaceKernel, P2PMatrixGenerator,
                            P2PMatrixSubsetGenerator)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs", 6650.0)
    rng = np.random.default_rng(15)
    pts = torch.as_tensor(rng.random((3, n)), device=dev)

    def tm(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = {}
    lap = P2PMatrixGenerator([LaplaceKernel(3)])
    ms = tm(lambda: lap(None, pts, pts, device=dev))
    gbs = 8.0 * n * n / (ms * 1e-3) / 1e9
    out["laplace_dense"] = {"shape": [n, n], "ms": ms, "GB_s": gbs, "frac_hbm": gbs / hbm}
    nh = n // 2
    hel = P2PMatrixGenerator([HelmholtzKernel(3)])
    ms = tm(lambda: hel(None, pts[:, :nh], pts[:, :nh], device=dev, k=10.0))
    gbs = 16.0 * nh * nh / (ms * 1e-3) / 1e9
    out["helmholtz_dense"] = {"shape": [nh, nh], "k": 10.0, "ms": ms, "GB_s": gbs,
                              "frac_hbm": gbs / hbm}
    it = torch.as_tensor(rng.integers(0, n, nsub), device=dev, dtype=torch.int32)
    js = torch.as_tensor(rng.integers(0, n, nsub), device=dev, dtype=torch.int32)
    sub = P2PMatrixSubsetGenerator([LaplaceKernel(3)])
    ms = tm(lambda: sub(None, pts, pts, tgtindices=it, srcindices=js, device=dev))
    out["laplace_subset"] = {"pairs": nsub, "ms": ms, "Gentries_s": nsub / (ms * 1e-3) / 1e9,
                             "GB_s_indices_and_result": 16.0 * nsub / (ms * 1e-3) / 1e9}
    out["peak_hbm_gbs"] = hbm
    return out


# FP64 operations per pair of the QBX applier's Laplace value (line Taylor,
# order p): a = c - s (3), |a|^2, a.b, |b|^2 (15), 1/|a| and 1/|a|^2 (3),
# w and v (2), 7 per recurrence step ((-(2n+1) w T_n - n v T_{n-1}) / (n+1),
# the sum), and the strength product and sum (2): 25 + 7 p.
def qbx_laplace_flops_per_pair(p):
    return 25 + 7 * p


def qbx_bench(dev, steps=5, warmup=3, ntheta=200, ntargets=20_000, order=12, k=2.5,
              cpu=True):
    """QBX layer potentials (sumpy.qbx.LayerPotential): single and double
    layer on the unit sphere, sources a Gauss-Legendre x midpoint quadrature
    (ntheta x 2 ntheta nodes, 80k at ntheta = 200), targets on the sphere
    with centers at depth 0.15 inside, line Taylor order 12, Laplace and
    Helmholtz (k = 2.5). Every target sums over every source (sumpy's
    direct applier). CUDA-event time per call, inputs resident; pairs per
    second, and for the Laplace value an FP64 rate against the measured
    DGEMM rate. The CPU leg times the oracle (numpy, one process) on 16
    targets against all sources."""
    import torch
    from sumpy_b200 import (DirectionalSourceDerivative, HelmholtzKernel, LaplaceKernel,
                            LayerPotential, LineTaylorLocalExpansion)
    from tests._pointsets import sphere_quadrature
    src_np, w_np = sphere_quadrature(ntheta)
    rng = np.random.default_rng(21)
    g = rng.standard_normal((3, ntargets))
    tgt_np = g / np.linalg.norm(g, axis=0)
    ctr_np = tgt_np * 0.85
    src, tgt, ctr = (torch.as_tensor(x, device=dev) for x in (src_np, tgt_np, ctr_np))
    dens = torch.as_tensor(w_np * src_np[2], device=dev)
    nsrc = src_np.shape[1]
    pairs = float(ntargets) * nsrc

    def tm(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = {"nsources": nsrc, "ntargets": ntargets, "order": order, "k": k}
    peaks = pipe_peaks_measured(dev)
    for name, base, kw in (("laplace", LaplaceKernel(3), {}),
                           ("helmholtz", HelmholtzKernel(3), {"k": k})):
        expn = LineTaylorLocalExpansion(base, order)
        s_lp = LayerPotential(expn, target_kernels=[base], source_kernels=[base], device=dev)
        d_lp = LayerPotential(expn, target_kernels=[base],
                              source_kernels=[DirectionalSourceDerivative(base, "normal")],
                              device=dev)
        d = dens if name == "laplace" else dens.to(torch.complex128)
        ms_s = tm(lambda: s_lp(None, tgt, src, ctr, [d], None, **kw))
        ms_d = tm(lambda: d_lp(None, tgt, src, ctr, [d], None, normal=src, **kw))
        out[name] = {"single_layer_ms": ms_s, "double_layer_ms": ms_d,
                     "single_layer_Gpairs_s": pairs / (ms_s * 1e-3) / 1e9,
                     "double_layer_Gpairs_s": pairs / (ms_d * 1e-3) / 1e9}
        if name == "laplace":
            tf = pairs * qbx_laplace_flops_per_pair(order) / (ms_s * 1e-3) / 1e12
            out[name]["single_layer_fp64_tflops"] = tf
            out[name]["frac_of_measured_dgemm"] = tf / peaks["fp64_tflops"]
    out["fp64_tflops_measured_dgemm"] = peaks["fp64_tflops"]
    if cpu:
        from oracle import qbx_oracle as Q
        sub = 16
        t0 = time.perf_counter()
        Q.lpot(order, Q.VALUE, tgt_np[:, :sub], ctr_np[:, :sub], src_np, w_np * src_np[2],
               scale=1 / (4 * np.pi), block=4)
        cpu_s = time.perf_counter() - t0
        out["cpu_oracle"] = {"kind": "port", "cores": 1, "sample": f"{sub} targets x {nsrc} "
                             "sources, Laplace single layer", "Gpairs_s":
                             sub * nsrc / cpu_s / 1e9}
    return out


def uniform_bench(dev, steps=5, warmup=3, n=20_000, order=6, cpu=True):
    """The reference's own CPU-runnable case: 20k sources and 20k separate
    targets U[0,1]^3 (seeds 15, 18; strengths seed 44), p = 6, max 30 per box,
    FP64 end to end. GPU time (CUDA events), accuracy against the FP64 GPU
    direct sum, and as its CPU baseline the oracle (C + OpenMP, all host
    threads) on the same tree."""
    import torch
    from sumpy_b200 import (P2P, LaplaceKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    src = np.random.default_rng(15).random((3, n))
    tgt = np.random.default_rng(18).random((3, n))
    q = np.random.default_rng(44).standard_normal(n)
    tree, trav, tcls = build_all(src, tgt, 30)
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    # replayed from a CUDA graph like the headline: at 20k points the eager
    # launch sequence is host-bound, and its timing drifts with the state the
    # earlier workloads leave in the process
    w = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                               translation_classes_data=tcls, device=dev, cuda_graph=True)
    qd = torch.as_tensor(q, device=dev)
    for _ in range(warmup):
        drive_fmm(None, w, [qd])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        (pot,) = drive_fmm(None, w, [qd])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    (ref,) = P2P([knl])(None, tgt, src, (q,), device=dev)
    out = {"workload": f"uniform {n} sources + {n} targets, p={order}, FP64", "launch": "CUDA graph replay",
           "ms_per_step": ms, "Mpts_s": n / (ms * 1e-3) / 1e6,
           "relL2_vs_direct": float((pot - ref).norm() / ref.norm())}
    if cpu:
        from oracle import oracle as O
        t0 = time.perf_counter()
        O.run_fmm(tree, trav, tcls, order, q)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"ms_per_step": 1e3 * dt, "cores": os.cpu_count(), "kind": "port",
                               "sample": "the same 20k + 20k evaluation, FP64 C/OpenMP oracle"}
        out["gpu_over_cpu"] = 1e3 * dt / ms
    return out


def helmholtz_bench(dev, steps=3, warmup=2, npoints=500_000, order=14, k=10.0,
                    precisions=("mixed", "fp64")):
    """3D Helmholtz (G = e^{ikr}/r, k = 10): 500k points on the unit sphere
    (sources = targets, exclude_self), strengths N(0,1) + i N(0,1), p = 14,
    max 32 per box. Mixed (complex64 near field on FP64 offsets, split-TF32
    M2L on the real embedding) and FP64 forms timed with CUDA events (L2
    flushed between steps); accuracy on 2,048 sampled targets against the
    complex128 GPU direct sum; per-stage times of the mixed form."""
    import torch
    from sumpy_b200 import (P2P, HelmholtzKernel, SumpyExpansionWrangler,
                            SumpyTreeIndependentDataForWrangler, drive_fmm)
    from sumpy_b200.expansion import (
        LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
        LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp)
    from sumpy_b200.tree import build_all
    rng = np.random.default_rng(2025)
    g = rng.standard_normal((3, npoints))
    pts = g / np.linalg.norm(g, axis=0)
    q = rng.standard_normal(npoints) + 1j * rng.standard_normal(npoints)
    t0 = time.perf_counter()
    tree, trav, tcls = build_all(pts, None, HELMHOLTZ_MAX_PARTICLES)
    t_tree = time.perf_counter() - t0
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    qd = torch.as_tensor(q, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn):
        for _ in range(warmup):
            fn()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record()
            fn()
            evs[i][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in evs) / steps

    smp = rng.choice(npoints, size=2048, replace=False)
    (ref,) = P2P([knl], exclude_self=True)(None, pts[:, smp], pts, (q,),
                                           target_to_source=smp, device=dev, k=k)
    ref = ref.cpu().numpy()
    out = {"workload": f"unit sphere n={npoints}, k={k}, p={order}, complex strengths, "
                       f"exclude_self, max {HELMHOLTZ_MAX_PARTICLES} per box",
           "tree_build_s": round(t_tree, 3), "m2l_entries": int(len(trav.from_sep_siblings_lists))}
    for precision in precisions:
        t0 = time.perf_counter()
        w = SumpyExpansionWrangler(ti, trav, np.complex128, lambda *a: order,
                                   kernel_extra_kwargs={"k": k}, translation_classes_data=tcls,
                                   precision=precision, device=dev)
        (pot,) = drive_fmm(None, w, [qd])
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        if precision == "mixed":
            from sumpy_b200.autotune import tune_m2l_item_groups
            tune_m2l_item_groups(w, lambda: drive_fmm(None, w, [qd]))
        ms = timed(lambda: drive_fmm(None, w, [qd]))
        w.check_status()
        got = pot.cpu().numpy()[smp]
        out[precision] = {"Mpts_s": npoints / (ms * 1e-3) / 1e6, "ms_per_step": ms,
                          "m2l_item_groups": w.m2l_item_groups,
                          "relL2_vs_direct": float(np.linalg.norm(got - ref) /
                                                   np.linalg.norm(ref)),
                          "setup_s": round(setup, 2)}
        if precision == "mixed":
            out["stage_ms_mixed"] = stage_breakdown(w, trav, qd, dev, roofline=False)[0]
            # adjoint with respect to the strengths: the FMM on the transposed
            # traversal (sumpy_b200.autograd.HelmholtzFMM's backward)
            from sumpy_b200.adjoint import transpose_traversal
            import gc
            # the eager launch sequence allocates per call: start from a
            # collected caching allocator, as the forward timing did
            gc.collect()
            torch.cuda.empty_cache()
            tree_t, trav_t, tcls_t = transpose_traversal(tree, trav, tcls)
            wa = SumpyExpansionWrangler(ti, trav_t, np.complex128, lambda *a: order,
                                        kernel_extra_kwargs={"k": k},
                                        translation_classes_data=tcls_t,
                                        precision=precision, device=dev)
            gd = pot.conj().contiguous()
            drive_fmm(None, wa, [gd])
            ms_adj = timed(lambda: drive_fmm(None, wa, [gd]))
            out["adjoint_forward_ratio_mixed"] = ms_adj / ms
            del wa
        del w
        torch.cuda.empty_cache()
    if "fp64" in out and "mixed" in out:
        out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def stage_breakdown(w, trav, q_dev, dev, roofline=True, pipe_peaks=None):
    """Per-stage device times of one FMM (CUDA events between the wrangler
    calls on the launching stream) and the roofline of the dominant stage."""
    import torch
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    def one_pass():
        ev = []

        def mark(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            ev.append((name, e))

        torch.cuda.synchronize()
        mark("start")
        qd = w.reorder_sources(q_dev)
        mark("reorder")
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
        mark("p2m")
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        mark("m2m")
        w.eval_direct(None, trav.target_boxes, trav.neighbor_source_boxes_starts,
                      trav.neighbor_source_boxes_lists, [qd])
        mark("p2p")
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                   mp)
        mark("m2l")
        w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                          trav.from_sep_smaller_by_level, mp)
        mark("m2p")
        pl = w.form_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                           trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                           trav.from_sep_bigger_lists, [qd])
        mark("p2l")
        loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                              trav.target_or_target_parent_boxes, loc + pl)
        mark("l2l")
        w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)
        mark("l2p")
        torch.cuda.synchronize()
        return {n1: e0.elapsed_time(e1) for (n0, e0), (n1, e1) in zip(ev, ev[1:])}

    # warm (clocks up after the host-side phases), then the per-stage median of 3 passes
    one_pass()
    passes = [one_pass() for _ in range(3)]
    stage = {k: float(np.median([ps[k] for ps in passes])) for k in passes[0]}
    if not roofline:
        return stage, None, None

    # algorithmic work per stage (the units the stage processes)
    tree = w.tree
    n = (w.level_orders[0] + 1) ** 2
    tb = trav.target_boxes
    ns = trav.neighbor_source_boxes_starts
    nl = trav.neighbor_source_boxes_lists
    cnt_t = tree.box_target_counts_nonchild[tb].astype(np.int64)
    src_per_list = np.add.reduceat(
        tree.box_source_counts_nonchild[nl].astype(np.int64), ns[:-1]) if len(nl) else 0
    empty = np.diff(ns) == 0
    src_per_list = np.where(empty, 0, src_per_list)
    pairs = int((cnt_t * src_per_list).sum()) - (tree.ntargets if tree.sources_are_targets else 0)
    m2l_entries = len(trav.from_sep_siblings_lists)
    m2p_pairs = 0
    for tbs, csr in zip(trav.target_boxes_sep_smaller_by_source_level,
                        trav.from_sep_smaller_by_level):
        if len(tbs):
            m2p_pairs += int((tree.box_target_counts_nonchild[np.asarray(tbs)].astype(np.int64)
                              * np.diff(np.asarray(csr.starts))).sum())
    mixed = w.precision == "mixed"
    kernels = {
        "m2l": (f"m2l_tc_kernel<{w.tc_format}>" if mixed else "m2l_f64_kernel<128>"),
        "m2p": "m2p_mixed_kernel<P>" if mixed else "m2p_reg_kernel<P>",
        "p2p": "p2p_csr_kernel<mixed>" if mixed else "p2p_csr_kernel<f64>",
        "p2l": "p2l_mixed_kernel<P>" if mixed else "p2l_reg_kernel<P>",
    }
    peak_bf16 = peaks.get("bf16_tflops", 1590.0)
    peak_hbm = peaks.get("hbm_gbs", 6650.0)
    src = "MEASURED_PEAKS.json (of measured)" if peaks else "fallback"

    def m2l_roof():
        ach = 2 * n * n * m2l_entries / (stage["m2l"] * 1e-3) / 1e12
        r = {"kernel": kernels["m2l"], "bound": "tensor", "achieved": ach, "peak": peak_bf16,
             "unit": "TFLOP/s", "frac": ach / peak_bf16, "traffic": None,
             "peak_source": "bf16_tflops " + src,
             "work": {"flops": 2 * n * n * m2l_entries, "entries": m2l_entries,
                      "per_unit": "2 n^2 flops per List-2 entry"}}
        if mixed:
            split = "row-scaled F16" if w.tc_format == "f16" else "TF32"
            r["note"] = (f"tcgen05 split-{split} GEMM (3 products); algorithmic flops = 2 n^2 "
                         "per List-2 entry (not the x3 split products, empty slots or padding); "
                         "the stage time includes the split pre-pass; peak: dense bf16 (the "
                         "f16 rate)")
        # dram__bytes_read.sum + dram__bytes_write.sum of this launch on the 1M-point
        # workload, one ncu capture per leaf size and operand format
        # (profiles/m2l_tc_f16_sphere_plummer_1M_p10.md, and for TF32
        # profiles/m2l_tf32x3_sphere_plummer_1M_p10.md)
        captured = ({96: 116.11e6 + 18.85e6} if w.tc_format == "f16"
                    else {32: 1.227e9 + 0.195e9, 96: 256.6e6 + 38.4e6})
        if mixed and tree.nsources == NPOINTS and n == (ORDER + 1) ** 2 and \
                MAX_PARTICLES in captured and \
                int(tree.box_source_counts_nonchild.max()) <= MAX_PARTICLES:
            r["traffic"] = captured[MAX_PARTICLES]
            r["traffic_unit"] = "bytes per launch (ncu capture)"
        return r

    # the dominant stage, with the stage's own roofline: M2L the tensor cores,
    # P2P the FP32 (mixed) / FP64 pipe, M2P and P2L HBM with 40 B per
    # evaluation (one target's or source's coordinates and value) -- they are
    # compute-bound at this order, so their FLOP/s against the measured
    # FP32/FP64 GEMM rate as well
    dom = max(("m2l", "m2p", "p2p", "p2l"), key=lambda k: stage[k])
    fp = pipe_peaks or {}
    if dom == "m2l":
        roof = m2l_roof()
    elif dom == "p2p":
        pk = fp.get("fp32_tflops" if mixed else "fp64_tflops")
        ach = 11 * pairs / (stage["p2p"] * 1e-3) / 1e12
        roof = {"kernel": kernels["p2p"], "bound": "fp32" if mixed else "fp64",
                "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": (ach / pk) if pk else None, "traffic": None,
                "peak_source": "torch.matmul FP32/FP64 GEMM measured in this run",
                "work": {"flops": 11 * pairs, "pairs": pairs, "per_unit": "11 flops per pair"}}
    else:
        units = m2p_pairs if dom == "m2p" else int(
            tree.box_source_counts_nonchild[np.asarray(trav.from_sep_bigger_lists)].sum())
        nbytes = 40 * units
        flops = units * 10 * n
        ach = nbytes / (stage[dom] * 1e-3) / 1e9
        pk = fp.get("fp32_tflops" if mixed else "fp64_tflops")
        ftf = flops / (stage[dom] * 1e-3) / 1e12
        roof = {"kernel": kernels[dom], "bound": "hbm", "achieved": ach, "peak": peak_hbm,
                "unit": "GB/s", "frac": ach / peak_hbm, "traffic": None,
                "peak_source": "hbm_gbs " + src,
                "work": {"bytes": nbytes, "evaluations": units,
                         "per_unit": "40 B per (target, List-3 box) / (List-4 source, box)"},
                "flops": {"achieved_tflops": ftf, "peak_tflops": pk,
                          "per_unit": "~10 n flops per evaluation",
                          "frac": (ftf / pk) if pk else None}}
    roof["dominant_stage"] = dom
    return stage, roof, m2l_roof()


def pipe_peaks_measured(dev):
    """FP32 and FP64 CUDA-core rates measured here: torch.matmul GEMMs with
    TF32 disabled (cuBLAS SGEMM / DGEMM), best of 5, CUDA events."""
    import torch
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for name, dt, m in (("fp32_tflops", torch.float32, 8192),
                            ("fp64_tflops", torch.float64, 4096)):
            a = torch.randn(m, m, device=dev, dtype=dt)
            b = torch.randn(m, m, device=dev, dtype=dt)
            torch.matmul(a, b)
            best = None
            for _ in range(5):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1)
                best = t if best is None else min(best, t)
            out[name] = 2.0 * m ** 3 / (best * 1e-3) / 1e12
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out


if __name__ == "__main__":
    main()
