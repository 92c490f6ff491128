#!/usr/bin/env python
"""Benchmark of the exact generalized winding number on B200 (one JSON line).

Workload (default): bumpy icosphere at subdivision 7, closed
(163,842 V, 327,680 F); 2^20 queries per GPU, half uniform in the 1.2x
bounding box and half within N(0, 1e-4) of the surface (seeded synthetic data;
no dataset exists for this path). A step is one pass of the hot path over that
batch: every (query, face) pair, 3.44e11 pairs per GPU.

Legs, all on the same inputs:
  * mixed  (headline when built): FP32 pair terms with compensated
    accumulation and FP64 refinement of near-surface pairs;
  * fp64:  the plain FP64 kernel, pair terms bit-identical to the reference;
  * fwdbwd_faces / fwdbwd_edges: mixed forward + the per-face mixed-precision
    adjoint / the mixed boundary-edge adjoint (both followed by the vertex gather);
  * adjoint_workloads: the same on the c3 mesh with 8% of its faces deleted and
    on the c3 mesh as a triangle soup (every edge a boundary edge);
  * c4: the gradient workload (subdivision-5 mesh, 8% faces deleted, 262,144
    near-surface queries): forward alone and forward + each adjoint;
  * c5: 64 uneven meshes in one persistent launch, forward alone and forward +
    boundary-edge adjoint replayed from one captured CUDA graph;
  * closest_point: the closest-point traversal beside the path
    (point_mesh_squared_distance over the median-split tree, bit-identical to
    the reference's CPU query) on the reference's own AABB benchmark shape
    (grid(350), 243,602 F x 10,000 points), on the c3 mesh x 2^20 queries and
    on grid(350) x 2^20 points: device time, end to end through the C ABI with
    host buffers, the oracle on this host's cores, and an exactness check;
  * vertex_normals: per-vertex normals (area weights) on the reference's
    benchmark shape (grid(350), 243,602 F) and on a subdivision-9 sphere
    (5,242,880 F): topology preparation once, then device time per evaluation
    with the achieved share of HBM bandwidth, end to end through the C ABI
    (preparation included), and the reference's serial CPU loop (the oracle);
  * fast_winding: the hierarchical approximation (Barill et al. 2018) on the
    headline workload at beta = 2 and 4: device time, end to end, max / p99
    error against the plain FP64 kernel's W, and the library's host evaluator
    on this host's cores.
`value` is whole-job pairs/s of the headline leg with inputs resident in HBM;
`e2e` is the same leg through the C ABI with pinned host buffers, the
host->device copies, device preprocessing and device->host copy inside the
timed region. L2 (126 MB) is flushed by a 256 MiB write before every timed
step. `cpu_baseline` times the oracle (CPU restatement of the reference's
Mojo kernel) on a bounded query sample on this host's cores.

Multi-GPU: `python -m torch.distributed.run --nproc-per-node N bench.py --gpus N`
shards nothing across ranks: each rank runs its own 2^20-query batch against
the same mesh (weak scaling, no data-path collective); the timed region is
bracketed by barriers and the slowest rank's time is reported.

`--impl reference` times the reference's CPU path (the oracle port, all host
threads) on a bounded sample of the same workload and prints the same metric.

`--case NAME [--case-queries N]` runs one kernel on a small case twice and
exits (the commands behind the ncu summaries in profiles/): fp64_c3 (streaming
FP64 kernel), fp64_tiled_c3 (FP64 over the prepared mesh), mixed_c3, adjoint_c4
(per-face mixed adjoint on the gradient workload), adjoint_c3 (the same on the
c3 workload), adjoint_soup (the same on the c3 triangle soup), edges_open_c3 (the
mixed boundary-edge adjoint on the open c3 mesh), welded_soup (the mixed edge adjoint
over the c3 soup's sides welded by position), closest_c3 (closest-point traversal), fwn_c3 (fast
winding number, beta = 2), normals_s9 (area-weighted vertex normals of the
subdivision-9 sphere) and batched_small (the batched persistent forward and
edge adjoint on 16 uneven meshes with at most 65,536 queries each).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mojo-libigl_b200", "python"))

METRIC = ("query·face pairs/s fwd & fwd+bwd, 327k F×1M Q, mixed vs FP64, "
          "≤1e-6 abs err")
FLOPS_PER_PAIR = 62  # algorithmic flops per pair, FMA = 2 (src/capi.mojo:218-235)
L2_FLUSH_BYTES = 256 << 20
KAPPA = 4.0  # refinement radius of the mixed leg, in face longest-edge units


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--queries", type=int, default=1 << 20, help="queries per GPU")
    p.add_argument("--subdivisions", type=int, default=7)
    p.add_argument("--legs", default="auto", help="comma list of mixed,fp64,fwdbwd")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-c4", action="store_true", help="skip the gradient workload")
    p.add_argument("--no-adjoint-workloads", action="store_true",
                   help="skip fwd+bwd on the open c3 mesh and the c3 triangle soup")
    p.add_argument("--no-c5", action="store_true", help="skip the batched workload")
    p.add_argument("--no-closest", action="store_true", help="skip the closest-point workloads")
    p.add_argument("--no-fast", action="store_true", help="skip the fast winding-number legs")
    p.add_argument("--no-normals", action="store_true", help="skip the vertex-normal workloads")
    p.add_argument("--case", choices=("fp64_c3", "fp64_tiled_c3", "mixed_c3", "adjoint_c4",
                                      "closest_c3", "fwn_c3", "normals_s9", "adjoint_c3",
                                      "adjoint_soup", "edges_open_c3", "welded_soup",
                                      "batched_small"),
                   help="run one kernel on a small case twice (for profiling) and exit")
    p.add_argument("--case-queries", type=int, default=None)
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="run the batched launch with the fixed default configuration instead "
                        "of the autotuner's choice (cached per GPU and size bucket)")
    return p.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def make_inputs(subdivisions: int, nq: int, rank: int):
    from igl import synthetic

    V, F = synthetic.bumpy_icosphere(subdivisions, seed=31)
    O = synthetic.mixed_queries(V, F, nq, seed=33 + 1000 * rank, near_sigma=1e-4)
    desc = (f"bumpy icosphere s={subdivisions} closed ({len(V)} V, {len(F)} F) x {nq} Q "
            "per GPU: 50% uniform in 1.2x bbox, 50% within N(0,1e-4) of the surface")
    return V, F, O, desc


def soa(V, F):
    return np.ascontiguousarray(V[F].transpose(1, 2, 0).reshape(9, len(F)))


# ---- CPU legs (oracle: only here, as the baseline and the reference arm) ----

def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_rate(tri, O, cores: int, target_s: float):
    """Pairs/s of the oracle on a query sample sized for about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # CPU restatement of the reference kernel (baseline only)

    nf = tri.shape[1]
    probe = O[: max(cores, 8)]
    t0 = time.perf_counter()
    oracle.winding_soa(tri, probe, workers=cores)
    rate = nf * len(probe) / max(time.perf_counter() - t0, 1e-6)
    n = int(min(len(O), max(cores, rate * target_s / nf)))
    # Same 50/50 box/near mix as the full batch: take from both halves.
    half = len(O) // 2
    sample = np.concatenate([O[: n // 2], O[half: half + n - n // 2]])
    t0 = time.perf_counter()
    oracle.winding_soa(tri, sample, workers=cores)
    dt = time.perf_counter() - t0
    return nf * len(sample) / dt, len(sample), dt


def oracle_isa() -> str:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle.isa()


def oracle_aabb_rate(P, V, F, tree, cores: int, target_s: float):
    """Points/s of the oracle's closest-point query over `cores` threads on a
    prefix of P sized to take about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    n = min(len(P), 4096)
    t0 = time.perf_counter()
    oracle.aabb_squared_distance(P[:n], V, F, tree=tree, workers=cores)
    dt = time.perf_counter() - t0
    n = int(min(len(P), max(n, n * target_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    oracle.aabb_squared_distance(P[:n], V, F, tree=tree, workers=cores)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def closest_point_workloads(nq: int):
    from igl import synthetic

    Vg, Fg = synthetic.terrain_grid(350)
    rng = np.random.default_rng(7)
    box = ([-10.0, -10.0, -5.0], [360.0, 360.0, 5.0])
    V3, F3, O3, _ = synthetic.workload("c3_mixed", n_queries=nq)
    return [
        ("reference_bench", "grid(350) height field (122,500 V, 243,602 F) x 10,000 points "
         "uniform in [-10,360]^2 x [-5,5] (the reference's AABB benchmark shape)",
         Vg, Fg, rng.uniform(*box, size=(10_000, 3))),
        ("c3", "c3 mesh (327,680 F, closed) x %d queries 50/50 box/near(1e-4)" % nq, V3, F3, O3),
        ("grid_1M", "grid(350) x %d points uniform in [-10,360]^2 x [-5,5]" % nq,
         Vg, Fg, rng.uniform(*box, size=(nq, 3))),
    ]


def host_closest_points(V, F, P):
    """This library's own CPU closest-point path at the reference's AABB
    benchmark shape, timed the way the reference times it: the tree prebuilt,
    the whole ``AABB.squared_distance`` call with the reference's worker policy,
    best of 3 after a warm-up. Reported beside the published 9.12 ms; a failure
    is recorded in the entry instead of ending the run."""
    try:
        import igl

        tree = igl.AABB()
        tree.init(V, F)
        tree.squared_distance(V, F, P)
        best = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            tree.squared_distance(V, F, P)
            best = min(best, time.perf_counter() - t0)
        depth = 1 + max(int(tree._tree[3]).bit_length(), 1)
        return {"ms": best * 1e3, "published_cpu_ms": 9.12,
                "workers": igl.worker_count(len(P), len(P) * len(F) * depth, "aabb"),
                "path": "igl.AABB.squared_distance, device='cpu' (mli_aabb_squared_distance "
                        "over the reference's span fan-out); the published figure is the "
                        "reference's README.md:105 on its own host"}
    except Exception as exc:  # informational field: never ends the bench
        return {"error": f"{type(exc).__name__}: {exc}"}


def reference_arm(args):
    """The reference's CPU path (the oracle port of its Mojo kernel, all host
    threads) on a fixed query sample of the headline workload; every step times
    the whole sample (wall clock), so ms_per_step is a measured step."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    V, F, O, desc = make_inputs(args.subdivisions, args.queries, 0)
    tri = soa(V, F)
    nf = len(F)
    cores = host_cores()
    rate, _, _ = oracle_rate(tri, O, cores, target_s=0.5)
    n = int(min(len(O), max(cores, rate * 2.5 / nf)))  # about 2.5 s per step
    half = len(O) // 2
    sample = np.concatenate([O[: n // 2], O[half: half + n - n // 2]])
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.winding_soa(tri, sample, workers=cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    dt = float(np.median(times))
    value = nf * len(sample) / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: " + desc,
        "config": {"workload": "c3: " + desc, "precision": "fp64 (reference CPU path)",
                   "faces": nf, "queries_per_gpu": args.queries,
                   "pairs_per_gpu_step": float(nf) * args.queries},
        "sample": {"queries_per_step": len(sample), "pairs_per_step": float(nf) * len(sample),
                   "step": "one pass of the reference CPU path over a fixed query sample of "
                           "the workload (50/50 box/near) against all faces, wall clock; "
                           "value = sample pairs / step time"},
        "cpu_baseline": {
            "value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
            "sample": f"{len(sample)} queries (50/50 box/near) x {nf} faces per step, oracle "
                      f"restatement of src/capi.mojo:205-294 over {cores} threads "
                      f"({cpu_model()}, {oracle.isa()} clone)",
        },
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU arm ----------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in out.strip().splitlines():
            parts = [x.strip() for x in row.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        load = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_arm(args):
    import torch

    from igl import _lib

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    handle = _lib.lib()
    V, F, O, desc = make_inputs(args.subdivisions, args.queries, rank)
    nf, nq = len(F), len(O)
    pairs = float(nf) * nq
    tri = soa(V, F)
    ld = nf + (nf & 1)
    dev = torch.device("cuda", local)
    tri_d = torch.zeros((9, ld), dtype=torch.float64, device=dev)
    tri_d[:, :nf] = torch.from_numpy(tri).to(dev)
    q_d = torch.from_numpy(O).to(dev)
    w_d = torch.empty(nq, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)

    def check(rc):
        if rc != 0:
            raise RuntimeError(_lib.last_error(handle))

    kernel_events = []  # (start, end) around the dominant kernel of each timed step
    refined_per_step = [0.0]

    def kernel_timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        kernel_events.append((e0, e1))

    def fp64_stream_step():
        kernel_timed(lambda: check(handle.wn_forward_fp64_device(
            tri_d.data_ptr(), ld, q_d.data_ptr(), w_d.data_ptr(), nf, nq, 0, sp)))

    # Mixed: the mesh is re-prepared from the FP64 soup and the queries are
    # re-sorted inside every step; the roofline times the pair kernel alone.
    mesh = ctypes.c_void_p()
    check(handle.wn_mixed_mesh_create(tri_d.data_ptr(), ld, nf, KAPPA, sp, ctypes.byref(mesh)))
    perm_d = torch.empty(nq, dtype=torch.int32, device=dev)
    wm_d = torch.empty(nq, dtype=torch.float64, device=dev)

    def fp64_step():
        # The fastest plain FP64 path: mesh re-prepared (strip-ordered tiles), then
        # the corner-reusing kernel; pair terms bit-identical to the reference.
        check(handle.wn_mixed_mesh_update(mesh, tri_d.data_ptr(), ld, sp))
        kernel_timed(lambda: check(handle.wn_forward_fp64_mesh_device(
            mesh, q_d.data_ptr(), nq, w_d.data_ptr(), sp)))

    def mixed_step():
        check(handle.wn_mixed_mesh_update(mesh, tri_d.data_ptr(), ld, sp))
        check(handle.wn_mixed_sort_queries(q_d.data_ptr(), nq, perm_d.data_ptr(), sp))
        kernel_timed(lambda: check(handle.wn_forward_mixed_sorted_device(
            mesh, q_d.data_ptr(), perm_d.data_ptr(), nq, wm_d.data_ptr(), sp)))

    # Forward + backward on the same batch, dL/dW ~ N(0, 1). "faces": the
    # per-face mixed-precision adjoint over the prepared mesh (queries re-sorted
    # inside), then the vertex gather. "edges": the boundary-edge adjoint (edge
    # list rebuilt from F inside the step), then the vertex gather.
    from igl import autograd as wa

    V_d = torch.from_numpy(V).to(dev)
    F_d = torch.from_numpy(F).to(dev)
    gw_d = torch.from_numpy(np.random.default_rng(7 + rank).normal(size=nq)).to(dev)
    dq_d = torch.empty((nq, 3), dtype=torch.float64, device=dev)
    dtri_d = torch.zeros_like(tri_d)

    def fwdbwd_faces_step():
        mixed_step()
        check(handle.wn_backward_mixed_device(mesh, q_d.data_ptr(), nq, gw_d.data_ptr(),
                                              dq_d.data_ptr(), dtri_d.data_ptr(), ld, sp))
        wa.gather_vertices(dtri_d, ld, nf, F_d, len(V))

    def fwdbwd_edges_step():
        mixed_step()
        wa.backward_edges(V_d, F_d, q_d, gw_d, precision="mixed")

    legs = {"mixed": mixed_step, "fp64": fp64_step, "fp64_stream": fp64_stream_step,
            "fwdbwd_faces": fwdbwd_faces_step, "fwdbwd_edges": fwdbwd_edges_step}
    headline = "mixed"
    wanted = ([k for k in legs if k != "fp64_stream"] if args.legs == "auto"
              else args.legs.split(","))
    if headline not in wanted:
        headline = wanted[0]

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(step, k, w):
        for _ in range(w):
            step()
        check(handle.wn_stream_check(sp))
        barrier()
        kernel_events.clear()
        handle.wn_mixed_stats(None, None, 1)  # reset the refinement counters
        launches0 = handle.wn_launch_count()
        events = []
        for _ in range(k):
            flush.fill_(1.0)  # 256 MiB write: evicts L2 between steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            events.append((e0, e1))
        barrier()
        check(handle.wn_stream_check(sp))
        launches = handle.wn_launch_count() - launches0
        refined = ctypes.c_int64(0)
        handle.wn_mixed_stats(ctypes.byref(refined), None, 1)
        refined_per_step[0] = refined.value / k
        total = sum(a.elapsed_time(b) for a, b in events) / 1e3
        kern = sum(a.elapsed_time(b) for a, b in kernel_events) / 1e3 / max(len(kernel_events), 1)
        if world > 1:
            t = torch.tensor([total, kern], dtype=torch.float64, device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            total, kern = float(t[0]), float(t[1])
        return total / k, launches, kern

    results = {}
    clocks = ClockSampler(local)
    for name in wanted:
        if name not in legs:
            continue
        if name == headline:
            clocks.start()
            results[name] = timed(legs[name], args.steps, max(args.warmup, 3))
            clock_info = clocks.stop()
            headline_refined = refined_per_step[0]
        else:
            results[name] = timed(legs[name], args.steps, 1)

    t_step, launches, t_kernel = results[headline]
    value = world * pairs / t_step
    fwdbwd = {}
    for name in ("fwdbwd_faces", "fwdbwd_edges"):
        if name in results:
            fwdbwd[name.split("_")[1]] = {
                "ms_per_step": results[name][0] * 1e3,
                "pairs_per_s": world * pairs / results[name][0],
                "ratio_to_forward": results[name][0] / t_step,
            }

    # Gradient workload: subdivision-5 mesh with 8% faces deleted (open), 262,144
    # near-surface queries: mixed forward alone vs forward + each adjoint.
    c4 = None
    if not args.no_c4:
        from igl import synthetic

        V4, F4, O4, desc4 = synthetic.workload("c4_grad")
        V4d, F4d = torch.from_numpy(V4).to(dev), torch.from_numpy(F4).to(dev)
        O4d = torch.from_numpy(O4).to(dev)
        g4d = torch.from_numpy(np.random.default_rng(47).normal(size=len(O4))).to(dev)
        tri4, ld4, nf4 = wa.triangle_soa(V4d, F4d)
        mesh4 = wa.PreparedMesh(tri4, ld4, nf4)

        def c4_fwd_w():
            check(handle.wn_mixed_mesh_update(mesh4.mesh, tri4.data_ptr(), ld4, sp))
            return mesh4.forward(O4d)

        def c4_fwd():
            c4_fwd_w()

        def c4_faces():
            c4_fwd()
            dq4, dt4 = mesh4.backward(O4d, g4d)
            wa.gather_vertices(dt4, ld4, nf4, F4d, len(V4))

        def c4_edges():
            c4_fwd()
            wa.backward_edges(V4d, F4d, O4d, g4d, precision="mixed")

        t4 = {k: timed(fn, args.steps, 2)[0] for k, fn in
              (("fwd", c4_fwd), ("faces", c4_faces), ("edges", c4_edges))}
        pairs4 = float(nf4) * len(O4)
        c4 = {"workload": desc4, "pairs": pairs4,
              "fwd_ms": t4["fwd"] * 1e3,
              "fwdbwd_faces_ms": t4["faces"] * 1e3, "fwdbwd_edges_ms": t4["edges"] * 1e3,
              "ratio_faces": t4["faces"] / t4["fwd"], "ratio_edges": t4["edges"] / t4["fwd"]}
        err4d = (c4_fwd_w() - wa.forward_fp64(tri4, ld4, nf4, O4d)).abs()
        c4["max_abs_err_vs_fp64"] = float(err4d.max())
        c4["p99_abs_err_vs_fp64"] = float(torch.quantile(err4d.float(), 0.99))
        # The same queries as float32 (BASELINE's "float32 and float64 points"): the
        # mixed forward and both adjoints take them as given; W's error is measured
        # against the plain FP64 kernel at the rounded points, over every query.
        O4f = O4d.to(torch.float32)
        O4r = O4f.to(torch.float64)

        def c4f_fwd():
            check(handle.wn_mixed_mesh_update(mesh4.mesh, tri4.data_ptr(), ld4, sp))
            return mesh4.forward(O4f)

        def c4f_faces():
            c4f_fwd()
            dq4, dt4 = mesh4.backward(O4f, g4d)
            wa.gather_vertices(dt4, ld4, nf4, F4d, len(V4))

        def c4f_edges():
            c4f_fwd()
            wa.backward_edges(V4d, F4d, O4f, g4d, precision="mixed")

        t4f = {k: timed(fn, args.steps, 2)[0] for k, fn in
               (("fwd", c4f_fwd), ("faces", c4f_faces), ("edges", c4f_edges))}
        err4 = (c4f_fwd() - wa.forward_fp64(tri4, ld4, nf4, O4r)).abs()
        c4["float32_queries"] = {
            "fwd_ms": t4f["fwd"] * 1e3, "fwdbwd_faces_ms": t4f["faces"] * 1e3,
            "fwdbwd_edges_ms": t4f["edges"] * 1e3,
            "ratio_faces": t4f["faces"] / t4f["fwd"], "ratio_edges": t4f["edges"] / t4f["fwd"],
            "max_abs_err_vs_fp64": float(err4.max()),
            "p99_abs_err_vs_fp64": float(torch.quantile(err4.float(), 0.99)),
            "queries_compared": len(O4)}
        mesh4.close()

    # fwd+bwd where the backward has work at the headline size: the c3 mesh with 8%
    # of its faces deleted (about 72k boundary edges) and the c3 mesh as a triangle
    # soup (every edge a boundary edge of the indexed mesh). Forward alone, then
    # forward + each adjoint + the vertex gather, dL/dW ~ N(0, 1).
    adj_work = None
    if not args.no_adjoint_workloads:
        from igl import synthetic

        adj_work = {}
        k_adj = min(args.steps, 3)
        for wname in ("c3_open", "c3_soup"):
            Va, Fa, Oa, desc_a = synthetic.workload(wname, n_queries=args.queries)
            Vad, Fad = torch.from_numpy(Va).to(dev), torch.from_numpy(Fa).to(dev)
            Oad = torch.from_numpy(Oa).to(dev)
            gad = torch.from_numpy(np.random.default_rng(57).normal(size=len(Oa))).to(dev)
            tria, lda, nfa = wa.triangle_soa(Vad, Fad)
            mesha = wa.PreparedMesh(tria, lda, nfa)

            def a_fwd():
                check(handle.wn_mixed_mesh_update(mesha.mesh, tria.data_ptr(), lda, sp))
                mesha.forward(Oad)

            def a_faces():
                a_fwd()
                dqa, dta = mesha.backward(Oad, gad)
                wa.gather_vertices(dta, lda, nfa, Fad, len(Va))

            def a_edges():
                a_fwd()
                wa.backward_edges(Vad, Fad, Oad, gad, precision="mixed")

            def a_edges64():
                a_fwd()
                wa.backward_edges(Vad, Fad, Oad, gad)

            def a_welded():
                a_fwd()
                wa.backward_welded_edges(Vad, Fad, Oad, gad)

            legs_a = [("fwd", a_fwd), ("faces", a_faces)]
            if wname == "c3_open":
                legs_a += [("edges", a_edges), ("edges_fp64", a_edges64)]
            else:
                legs_a += [("welded", a_welded)]
            ta = {k: timed(fn, k_adj, 1)[0] for k, fn in legs_a}
            _, ne_a, _ = wa.boundary_edges(Vad, Fad)
            adj_work[wname] = {
                "workload": desc_a, "pairs": float(nfa) * len(Oa), "boundary_edges": ne_a,
                "fwd_ms": ta["fwd"] * 1e3, "fwdbwd_faces_ms": ta["faces"] * 1e3,
                "ratio_faces": ta["faces"] / ta["fwd"],
                "steps": k_adj,
                "note": "faces: per-face mixed adjoint; edges: mixed boundary-edge adjoint; "
                        "welded: the soup's sides welded by position, mixed edge adjoint "
                        "(welding inside the step)"}
            for leg in ("edges", "welded"):
                if leg in ta:
                    adj_work[wname][f"fwdbwd_{leg}_ms"] = ta[leg] * 1e3
                    adj_work[wname][f"ratio_{leg}"] = ta[leg] / ta["fwd"]
            if "edges_fp64" in ta:
                adj_work[wname]["fwdbwd_edges_fp64_ms"] = ta["edges_fp64"] * 1e3
                adj_work[wname]["ratio_edges_fp64"] = ta["edges_fp64"] / ta["fwd"]
            mesha.close()
            del Vad, Fad, Oad, gad, tria

    # Batched workload: 64 bumpy icospheres (subdivision U{2..7}, 0-10% faces
    # deleted, queries log-uniform in [1024, 2^20]), forward and forward +
    # boundary-edge adjoint as one captured CUDA graph of persistent launches.
    c5 = None
    if not args.no_c5:
        from igl import autotune, batched, synthetic

        work = synthetic.batched_workload(seed=51 + rank)
        meshes = [(Vm, Fm) for Vm, Fm, _ in work]
        queries = [Om for _, _, Om in work]
        t_tune = time.perf_counter()
        tuned = autotune.tune(meshes, queries) if args.autotune else None
        t_tune = time.perf_counter() - t_tune
        cfg = tuned["config"] if tuned else {"qpt": 2, "target_pairs": 1 << 21, "kappa": 4.0}
        bt = batched.Batch(meshes, queries, **cfg)
        bt.gW.normal_()
        t_f = timed(lambda: bt.forward(), args.steps, 2)[0]
        # Accuracy of the chosen configuration: up to 128 queries of every mesh
        # against the plain FP64 kernel.
        W_b = bt.split(bt.forward().clone())
        err_b = []
        for (Vm, Fm), Om, wm in zip(meshes, queries, W_b):
            sel = np.random.default_rng(len(Om)).choice(len(Om), min(len(Om), 128), replace=False)
            tri_m, ld_m, nf_m = wa.triangle_soa(torch.from_numpy(Vm).to(dev),
                                                torch.from_numpy(Fm).to(dev))
            ref_m = wa.forward_fp64(tri_m, ld_m, nf_m, torch.from_numpy(Om[sel]).to(dev))
            err_b.append(float((wm[torch.from_numpy(sel).to(dev)] - ref_m).abs().max()))
        bt.capture(backward=True)
        t_g, launches_g, _ = timed(bt.replay, args.steps, 2)
        info_b = bt.info()
        # The same graph with the FP64 adjoint, for comparison.
        bt.graph = None
        torch.cuda.synchronize()
        bt.handle.wn_batch_set_adjoint_fp64(bt.batch, 1)
        bt.capture(backward=True)
        t_g64 = timed(bt.replay, args.steps, 2)[0]
        c5 = {"workload": "64 bumpy icospheres, subdivision U{2..7}, 0-10% faces deleted, "
                          "queries log-uniform in [1024, 2^20], 50/50 box/near(1e-3)",
              "meshes": len(meshes), "pairs": bt.pairs, "config": cfg,
              "autotuned": tuned is not None,
              "autotune": ({k: v for k, v in tuned.items() if k != "config"} | {"seconds": t_tune}
                           if tuned else None),
              "info": info_b,
              "fwd_ms": t_f * 1e3, "fwd_pairs_per_s": world * bt.pairs / t_f,
              "graph_fwdbwd_ms": t_g * 1e3, "graph_fwdbwd_pairs_per_s": world * bt.pairs / t_g,
              "ratio_fwdbwd_to_fwd": t_g / t_f,
              "adjoint": "mixed (per-mesh Morton-ordered 64-edge tiles, FP64 near pairs)",
              "graph_fwdbwd_fp64_adjoint_ms": t_g64 * 1e3,
              "ratio_fwdbwd_fp64_adjoint": t_g64 / t_f,
              "max_abs_err_vs_fp64": max(err_b),
              "error_sample": "up to 128 queries of each mesh against the plain FP64 kernel"}
        bt.close()

    # The reference's own winding-number benchmark (bench/bench.py:96-112 there):
    # grid(120) = 28,322 faces, 256 and then 1024 queries drawn from
    # default_rng(0) in [0,119]^2 x [-2,2], each call timed as it does (wall
    # clock, best of 3 after one warm-up) through the drop-in igl.winding_number.
    refwn = None
    if rank == 0:
        import igl
        from igl import synthetic

        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        WV, WF = synthetic.terrain_grid(120)
        rng_w = np.random.default_rng(0)
        Q256 = rng_w.uniform([0, 0, -2], [119, 119, 2], size=(256, 3))
        Q1024 = rng_w.uniform([0, 0, -2], [119, 119, 2], size=(1024, 3))

        def best_of(fn, repeat=3):
            fn()
            best = float("inf")
            for _ in range(repeat):
                t0 = time.perf_counter()
                fn()
                best = min(best, time.perf_counter() - t0)
            return best * 1e3

        W_gpu = igl.winding_number(WV, WF, Q1024, device="gpu")
        W_ref = oracle.winding_number(WV, WF, Q1024, workers=host_cores())
        refwn = {
            "workload": "grid(120) height field (14,400 V, 28,322 F); 256 and 1024 queries "
                        "uniform in [0,119]^2 x [-2,2] from default_rng(0) (the reference's "
                        "winding-number benchmark)",
            "gpu_1024q_ms": best_of(lambda: igl.winding_number(WV, WF, Q1024, device="gpu")),
            "published_gpu_1024q_ms": 53.47,
            "cpu_256q_ms": best_of(lambda: igl.winding_number(WV, WF, Q256)),
            "published_cpu_256q_ms": 60.66,
            "cpu_1024q_ms": best_of(lambda: igl.winding_number(WV, WF, Q1024)),
            "published_cpu_1024q_ms": 215.09,
            "cpu_workers": igl.worker_count(len(Q1024), len(WF) * len(Q1024), "winding"),
            "oracle_port_1024q_ms": best_of(
                lambda: oracle.winding_number(WV, WF, Q1024, workers=min(4, host_cores()))),
            "oracle_port_workers": min(4, host_cores()),
            "max_abs_diff_gpu_vs_oracle": float(np.abs(W_gpu - W_ref).max()),
            "note": "wall clock of the whole API call (validation, SoA repack, copies, launch); "
                    "published figures from the reference's README.md:93-104 (Xeon E5-2697 v4 "
                    "host, GPU model not stated); the CPU rows run this library's host path "
                    "with the reference's worker policy on this machine's cores",
        }
        # The two plain-FP64 configurations through the drop-in, end to end (host
        # arrays in, host W out): 1,280 F x 4,096 Q and 18,842 F x 2^20 Q.
        for name in ("c1_cpu", "c2_open"):
            Vd, Fd, Od, desc_d = synthetic.workload(name)
            pairs_d = float(len(Fd)) * len(Od)
            W_d = igl.winding_number(Vd, Fd, Od, device="gpu")
            sub = np.random.default_rng(8).choice(len(Od), min(len(Od), 512), replace=False)
            entry = {"workload": desc_d, "pairs": pairs_d,
                     "gpu_ms": best_of(lambda: igl.winding_number(Vd, Fd, Od, device="gpu")),
                     "max_abs_diff_vs_oracle_512q": float(np.abs(
                         W_d[sub] - oracle.winding_number(Vd, Fd, Od[sub],
                                                          workers=host_cores())).max())}
            entry["gpu_pairs_per_s"] = pairs_d / (entry["gpu_ms"] * 1e-3)
            if name == "c1_cpu":
                entry["cpu_ms"] = best_of(lambda: igl.winding_number(Vd, Fd, Od))
                entry["cpu_workers"] = igl.worker_count(len(Od), pairs_d, "winding")
            refwn["drop_in_" + name] = entry

    # Closest points (the AABB query beside the winding number).
    closest = None
    if not args.no_closest:
        from igl import distance

        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        closest = {}
        for key, desc_c, Vc, Fc, Pc in closest_point_workloads(args.queries):
            tree = distance.DeviceAABB(Vc, Fc)
            P_d = torch.from_numpy(Pc).to(dev)
            npc = len(Pc)
            s_d = torch.empty(npc, dtype=torch.float64, device=dev)
            i_d = torch.empty(npc, dtype=torch.int64, device=dev)
            c_d = torch.empty((npc, 3), dtype=torch.float64, device=dev)

            def aabb_step():
                kernel_timed(lambda: check(handle.wn_aabb_squared_distance_device(
                    tree.tree, P_d.data_ptr(), npc, s_d.data_ptr(), i_d.data_ptr(),
                    c_d.data_ptr(), sp)))

            t_c, launches_c, t_ck = timed(aabb_step, max(args.steps, 5), 3)
            entry = {"workload": desc_c, "faces": len(Fc), "points": npc,
                     "ms_per_step": t_c * 1e3, "kernel_ms": t_ck * 1e3,
                     "points_per_s": world * npc / t_c, "gpu_launches_per_step": launches_c /
                     max(args.steps, 5)}
            # End to end: pinned host points in, host results out (C ABI).
            P_h = torch.from_numpy(Pc).pin_memory()
            s_h = torch.empty(npc, dtype=torch.float64).pin_memory()
            i_h = torch.empty(npc, dtype=torch.int64).pin_memory()
            c_h = torch.empty((npc, 3), dtype=torch.float64).pin_memory()

            def host_call():
                check(handle.wn_aabb_squared_distance_host(tree.tree, P_h.data_ptr(), npc,
                                                           s_h.data_ptr(), i_h.data_ptr(),
                                                           c_h.data_ptr()))

            if not args.no_e2e:
                host_call()
                barrier()
                reps = max(args.steps, 5)
                t0 = time.perf_counter()
                for _ in range(reps):
                    host_call()
                dt_e = (time.perf_counter() - t0) / reps
                entry["e2e"] = {"value": world * npc / dt_e, "unit": "points/s",
                                "ms_per_step": dt_e * 1e3, "h2d_bytes_per_step": int(Pc.nbytes),
                                "d2h_bytes_per_step": int(npc * 40),
                                "path": "wn_aabb_squared_distance_host (C ABI, pinned host buffers)"}
            if rank == 0:
                torch.cuda.synchronize()
                idx = np.random.default_rng(3).choice(npc, min(npc, 2048), replace=False)
                exp = oracle.aabb_squared_distance(Pc[idx], Vc, Fc, tree=tree.tree_arrays,
                                                   workers=host_cores())
                got = (s_d.cpu().numpy()[idx], i_d.cpu().numpy()[idx], c_d.cpu().numpy()[idx])
                entry["exact_vs_oracle_2048_points"] = all(
                    np.array_equal(g, e) for g, e in zip(got, exp))
                if world == 1 and not args.no_cpu_baseline:
                    cores = host_cores()
                    rate, n_s, dt_s = oracle_aabb_rate(Pc, Vc, Fc, tree.tree_arrays, cores, 4.0)
                    entry["cpu_baseline"] = {
                        "value": rate, "unit": "points/s", "cores": cores, "kind": "port",
                        "sample": f"first {n_s} points in {dt_s:.1f} s, oracle restatement of "
                                  f"src/capi.mojo:401-586 over {cores} threads"}
                if key == "reference_bench":
                    entry["host_path"] = host_closest_points(Vc, Fc, Pc)
            if key == "c3":
                # Signed distance: traversal + winding-number sign, all on the device.
                S_d = torch.empty(npc, dtype=torch.float64, device=dev)
                W_d = torch.empty(npc, dtype=torch.float64, device=dev)
                fwn_s = tree.fast_winding()

                def signed_step():
                    kernel_timed(lambda: check(handle.wn_signed_distance_fast_device(
                        tree.tree, fwn_s._handle, 2.0, P_d.data_ptr(), npc, S_d.data_ptr(),
                        i_d.data_ptr(), c_d.data_ptr(), W_d.data_ptr(), sp)))

                t_s = timed(signed_step, max(args.steps, 5), 3)[0]
                entry["signed_distance_fast"] = {
                    "ms_per_step": t_s * 1e3, "points_per_s": world * npc / t_s,
                    "note": "closest point and fast winding number (beta = 2) side by side on two "
                            "streams from one Morton order, then the sign"}
            closest[key] = entry
            tree.close()
        closest["note"] = ("reference's published AABB.squared_distance for the "
                           "reference_bench shape: 9.12 ms (its own host, README.md:105)")

    # Per-vertex normals (area weights): prepared topology, then one launch per call.
    normals_out = None
    if not args.no_normals:
        from igl import normals as wnorm
        from igl import synthetic

        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        normals_out = {}
        hbm = None
        peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(peaks):
            hbm = json.load(open(peaks)).get("hbm_gbs")
        meshes = [("reference_bench", "grid(350) height field (122,500 V, 243,602 F), area "
                   "weights (the reference's per_vertex_normals benchmark shape)",
                   *synthetic.terrain_grid(350)),
                  ("s9", "bumpy icosphere s=9 (2,621,442 V, 5,242,880 F), area weights",
                   *synthetic.bumpy_icosphere(9, seed=91))]
        for key, desc_n, Vn, Fn in meshes:
            nvn, nfn = len(Vn), len(Fn)
            t0 = time.perf_counter()
            dn = wnorm.DeviceNormals(Fn, nvn)
            torch.cuda.synchronize()
            t_prep = time.perf_counter() - t0
            Vn_d = torch.from_numpy(Vn).to(dev)
            Nn_d = torch.empty((nvn, 3), dtype=torch.float64, device=dev)

            def normals_step():
                kernel_timed(lambda: check(handle.wn_vertex_normals_device(
                    dn.h, Vn_d.data_ptr(), 1, Nn_d.data_ptr(), sp)))

            t_n, launches_n, t_nk = timed(normals_step, max(args.steps, 5), 3)
            # Algorithmic bytes: V and N (24 B per vertex each), int32 faces (12 B per
            # face), the vertex -> (face, corner) lists (4 B per vertex + 12 B per face).
            alg = 52 * nvn + 24 * nfn + 4
            entry = {"workload": desc_n, "vertices": nvn, "faces": nfn,
                     "prepare_topology_ms": t_prep * 1e3,
                     "ms_per_step": t_n * 1e3, "kernel_ms": t_nk * 1e3,
                     "vertices_per_s": world * nvn / t_n,
                     "roofline": {"bound": "hbm", "algorithmic_bytes": alg,
                                  "achieved": alg / t_nk / 1e9, "peak": hbm, "unit": "GB/s",
                                  "frac": (alg / t_nk / 1e9 / hbm) if hbm else None,
                                  "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}}
            Nd = Nn_d.cpu().numpy()
            host = np.zeros_like(Vn)
            t0 = time.perf_counter()
            handle.mli_vertex_normals(Vn.ctypes.data, Fn.ctypes.data, host.ctypes.data, nvn, nfn, 1)
            dt_host = time.perf_counter() - t0
            entry["bit_identical_to_host_path"] = Nd.tobytes() == host.tobytes()
            entry["host_path_ms"] = dt_host * 1e3
            if not args.no_e2e:
                V_h = torch.from_numpy(Vn).pin_memory()
                N_h = torch.empty((nvn, 3), dtype=torch.float64).pin_memory()
                call = lambda: check(handle.wn_vertex_normals_host(  # noqa: E731
                    V_h.data_ptr(), nvn, Fn.ctypes.data, nfn, 1, N_h.data_ptr()))
                call()
                reps = 3
                t0 = time.perf_counter()
                for _ in range(reps):
                    call()
                dt_e = (time.perf_counter() - t0) / reps
                entry["e2e"] = {"value": world * nvn / dt_e, "unit": "vertices/s",
                                "ms_per_step": dt_e * 1e3,
                                "h2d_bytes_per_step": int(Vn.nbytes + Fn.nbytes),
                                "d2h_bytes_per_step": int(nvn * 24),
                                "path": "wn_vertex_normals_host (C ABI, one shot: faces "
                                        "validated and prepared inside the timed region)"}
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                t0 = time.perf_counter()
                oracle.per_vertex_normals(Vn, Fn, 1)
                dt_o = time.perf_counter() - t0
                entry["cpu_baseline"] = {"value": nvn / dt_o, "unit": "vertices/s", "cores": 1,
                                         "kind": "port", "ms": dt_o * 1e3,
                                         "sample": "whole mesh, the oracle restatement of "
                                                   "src/capi.mojo:146-202 (serial, as the "
                                                   "reference's loop)"}
            normals_out[key] = entry
            dn.close()
        normals_out["note"] = ("reference's published per_vertex_normals (area, 243.6k F): "
                               "6.15 ms on its own host (README.md:101)")

    # Fast (hierarchical) winding numbers on the headline workload.
    fast = None
    if not args.no_fast:
        import igl

        fwn = igl.FastWindingNumber(V, F)
        wf_d = torch.empty(nq, dtype=torch.float64, device=dev)
        fast = {"workload": "c3: " + desc, "tree": fwn.info(),
                "note": "error against the plain FP64 kernel's W on every query"}
        have_exact = "fp64" in results
        for beta in (2.0, 4.0):
            def fast_step(beta=beta):
                kernel_timed(lambda: check(handle.wn_fast_eval_device(
                    fwn._handle, q_d.data_ptr(), nq, beta, wf_d.data_ptr(), sp)))

            t_f, launches_f, t_fk = timed(fast_step, max(args.steps, 5), 3)
            entry = {"ms_per_step": t_f * 1e3, "kernel_ms": t_fk * 1e3,
                     "queries_per_s": world * nq / t_f,
                     "pair_equivalent_per_s": world * pairs / t_f,
                     "speedup_vs_exact_mixed": (results["mixed"][0] / t_f
                                                if "mixed" in results else None)}
            if have_exact:
                err = (wf_d - w_d).abs()
                entry["max_abs_err_vs_fp64"] = float(err.max())
                entry["p99_abs_err_vs_fp64"] = float(torch.quantile(err.float(), 0.99))
            if not args.no_e2e:
                q_h = torch.from_numpy(O).pin_memory()
                w_h = torch.empty(nq, dtype=torch.float64).pin_memory()
                call = lambda beta=beta: check(handle.wn_fast_eval_host(  # noqa: E731
                    fwn._handle, q_h.data_ptr(), nq, beta, w_h.data_ptr()))
                call()
                barrier()
                t0 = time.perf_counter()
                for _ in range(max(args.steps, 5)):
                    call()
                dt = (time.perf_counter() - t0) / max(args.steps, 5)
                entry["e2e"] = {"value": world * nq / dt, "unit": "queries/s",
                                "ms_per_step": dt * 1e3, "h2d_bytes_per_step": int(O.nbytes),
                                "d2h_bytes_per_step": int(nq * 8),
                                "path": "wn_fast_eval_host (C ABI, pinned host buffers)"}
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                cores = host_cores()
                n_s = min(nq, 1 << 18)
                w_s = np.empty(n_s)
                O_s = np.ascontiguousarray(O[:n_s])
                t0 = time.perf_counter()
                fn = handle.wn_fast_eval_cpu
                from concurrent.futures import ThreadPoolExecutor

                parts = [(i * n_s // cores, (i + 1) * n_s // cores) for i in range(cores)]
                with ThreadPoolExecutor(cores) as pool:
                    list(pool.map(lambda ab, beta=beta: fn(fwn._handle, O_s.ctypes.data, n_s,
                                                           beta, w_s.ctypes.data, ab[0], ab[1]),
                                  parts))
                dt = time.perf_counter() - t0
                entry["cpu_host_evaluator"] = {
                    "value": n_s / dt, "unit": "queries/s", "cores": cores,
                    "sample": f"first {n_s} queries in {dt:.2f} s (wn_fast_eval_cpu spans)"}
            fast[f"beta_{beta:g}"] = entry
        fwn.close()

    # Accuracy of the mixed leg against the FP64 kernel on every query.
    accuracy = None
    if "mixed" in results and "fp64" in results:
        err = (wm_d - w_d).abs()
        accuracy = {"max_abs_err_vs_fp64": float(err.max()),
                    "p99_abs_err_vs_fp64": float(torch.quantile(err.float(), 0.99)),
                    "queries_compared": nq}

    # Parity spot check in the same run: fp64 GPU vs the oracle on 128 queries.
    parity = None
    if rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        fp64_step()
        torch.cuda.synchronize()
        w_gpu = w_d.cpu().numpy()
        idx = np.concatenate([np.arange(64), nq // 2 + np.arange(64)])
        ref = oracle.winding_soa(tri, O[idx], workers=host_cores())
        parity = float(np.abs(w_gpu[idx] - ref).max())

    # Roofline of the dominant kernel: algorithmic flops per launch / duration.
    bits = 32 if headline == "mixed" else 64
    peak = ctypes.c_double(0.0)
    check(handle.wn_probe_fma_tflops(bits, ctypes.byref(peak)))
    achieved = FLOPS_PER_PAIR * pairs / t_kernel / 1e12
    kname = "mixed_forward_kernel" if headline == "mixed" else "fp64_tiled_kernel"
    traffic = None
    traffic_file = os.path.join(ROOT, "profiles", "dram_traffic_full_size.txt")
    if os.path.exists(traffic_file) and nf == 327680 and nq == 1 << 20:
        for line in open(traffic_file):
            parts = line.split()
            if len(parts) == 4 and parts[0] == kname:
                traffic = int(parts[1]) + int(parts[2])
    roofline = {
        "bound": f"fp{bits}", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
        "frac": achieved / peak.value if peak.value else None, "traffic": traffic,
        "kernel": kname, "kernel_ms": t_kernel * 1e3,
        "traffic_source": "profiles/dram_traffic_full_size.txt (one-pass ncu capture of the "
                          "same kernel at this size)" if traffic else None,
        "peak_source": f"measured live on this GPU: FP{bits} FMA-chain probe "
                       "(wn_probe_fma_tflops), FMA = 2 flops",
        "flops_per_pair": FLOPS_PER_PAIR,
    }

    # End to end through the C ABI with pinned host buffers: H2D of the soup
    # and the queries, mesh preparation, query sort, kernel, D2H of W.
    e2e = None
    if not args.no_e2e:
        tri_h = torch.from_numpy(tri).pin_memory()
        q_h = torch.from_numpy(O).pin_memory()
        w_h = torch.empty(nq, dtype=torch.float64).pin_memory()
        if headline == "mixed":
            call = lambda: check(handle.wn_forward_mixed_host(  # noqa: E731
                tri_h.data_ptr(), q_h.data_ptr(), w_h.data_ptr(), nf, nq, KAPPA))
            path = "wn_forward_mixed_host (C ABI, pinned host buffers)"
        else:
            call = lambda: check(handle.wn_forward_fp64_host(  # noqa: E731
                tri_h.data_ptr(), q_h.data_ptr(), w_h.data_ptr(), nf, nq, 0))
            path = "wn_forward_fp64_host (C ABI, pinned host buffers)"
        call()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            call()
        dt = (time.perf_counter() - t0) / args.steps
        if world > 1:
            t = torch.tensor([dt], dtype=torch.float64, device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            dt = float(t.item())
        e2e = {"value": world * pairs / dt, "unit": "pairs/s",
               "h2d_bytes_per_step": int(tri.nbytes + O.nbytes), "d2h_bytes_per_step": int(nq * 8),
               "path": path}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        rate, n, dt = oracle_rate(tri, O, cores, target_s=12.0)
        cpu = {"value": rate, "unit": "pairs/s", "cores": cores, "kind": "port",
               "sample": f"{n} queries (50/50 box/near) x {nf} faces in {dt:.1f} s, oracle "
                         f"restatement of src/capi.mojo:205-294 over {cores} threads "
                         f"({cpu_model()}, {oracle_isa()} clone)"}
        # The reference's own fan-out caps its pool at four workers (python/igl/_lib.py:37).
        w4 = min(4, cores)
        rate4, n4, dt4 = oracle_rate(tri, O, w4, target_s=6.0)
        cpu["reference_fanout"] = {"value": rate4, "unit": "pairs/s", "cores": w4,
                                   "sample": f"{n4} queries in {dt4:.1f} s over {w4} threads, "
                                             "the reference's MAX_WORKERS"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if headline == "mixed" else "f64", "data": "synthetic: " + desc,
            "config": {"workload": "c3: " + desc, "precision": headline, "faces": nf,
                       "kappa": KAPPA if headline == "mixed" else None,
                       "queries_per_gpu": nq, "pairs_per_gpu_step": pairs,
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"query batches per GPU, {world} GPU(s)"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clock_info,
            "legs": {k: {"pairs_per_s": world * pairs / v[0], "ms_per_step": v[0] * 1e3,
                         "kernel_ms": v[2] * 1e3} for k, v in results.items()},
            "mixed_over_fp64": (results["fp64"][0] / results["mixed"][0]
                                if "mixed" in results and "fp64" in results else None),
            "fwd_bwd": fwdbwd,
            "c4_fwd_bwd": c4,
            "adjoint_workloads": adj_work,
            "c5_batched": c5,
            "winding_reference_bench": refwn,
            "closest_point": closest,
            "fast_winding": fast,
            "vertex_normals": normals_out,
            "accuracy": accuracy,
            "refinement": ({"pairs_refined_fp64_per_step": headline_refined,
                            "fraction": headline_refined / pairs}
                           if headline == "mixed" else None),
            "fp64_vs_oracle_max_abs_err_128q": parity,
        }
        print(json.dumps(line), flush=True)
    handle.wn_mixed_mesh_destroy(mesh)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_case(args):
    """One kernel, twice, on a reduced query batch of the c3 (or c4) workload."""
    import torch

    if args.case == "batched_small":
        from igl import batched, synthetic

        work = synthetic.batched_workload(n_meshes=16, seed=51, max_queries=1 << 16, max_level=6)
        bt = batched.Batch([(Vm, Fm) for Vm, Fm, _ in work], [Om for _, _, Om in work])
        bt.gW.normal_()
        for _ in range(2):
            bt.forward()
            bt.backward()
        torch.cuda.synchronize()
        print("ok", args.case, bt.info(), float(bt.W.abs().sum()))
        bt.close()
        return

    if args.case == "edges_open_c3":
        from igl import autograd as wa
        from igl import synthetic

        V, F, O, _ = synthetic.workload("c3_open", n_queries=args.case_queries or 65536)
        Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
        g = torch.from_numpy(np.random.default_rng(5).normal(size=len(O))).cuda()
        edges = wa.boundary_edges(Vt, Ft)
        for _ in range(2):
            dV, dq = wa.backward_edges(Vt, Ft, Ot, g, edges, precision="mixed")
        torch.cuda.synchronize()
        print("ok", args.case, edges[1], len(O), float(dq.abs().sum()))
        return

    if args.case == "welded_soup":
        from igl import autograd as wa
        from igl import synthetic

        V, F, O, _ = synthetic.workload("c3_soup", n_queries=args.case_queries or 65536)
        Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
        g = torch.from_numpy(np.random.default_rng(5).normal(size=len(O))).cuda()
        welded = wa.welded_edges(Vt, Ft)
        for _ in range(2):
            dV, dq = wa.backward_welded_edges(Vt, Ft, Ot, g, welded)
        torch.cuda.synchronize()
        print("ok", args.case, welded[1], len(O), float(dV.abs().sum()), float(dq.abs().sum()))
        return

    if args.case == "normals_s9":
        from igl import normals, synthetic

        V, F = synthetic.bumpy_icosphere(9, seed=91)
        dn = normals.DeviceNormals(F, len(V))
        Vt = torch.from_numpy(V).cuda()
        for _ in range(2):
            N = dn.evaluate(Vt, 1)
        torch.cuda.synchronize()
        dn.close()
        print("ok", args.case, len(F), len(V), float(N.abs().sum()))
        return

    from igl import _lib, distance, synthetic
    from igl import autograd as wa

    handle = _lib.lib()
    default_nq = {"fp64_c3": 16384, "fp64_tiled_c3": 32768, "mixed_c3": 65536,
                  "adjoint_c4": 16384, "closest_c3": 1 << 20, "fwn_c3": 1 << 20,
                  "normals_s9": 1, "adjoint_c3": 65536, "adjoint_soup": 65536}[args.case]
    nq = args.case_queries or default_nq
    wl = {"adjoint_c4": "c4_grad", "adjoint_soup": "c3_soup"}.get(args.case, "c3_mixed")
    V, F, O, _ = synthetic.workload(wl, n_queries=nq)
    if args.case in ("adjoint_c3", "adjoint_soup"):
        args.case = "adjoint_c4"  # the same call on the c3 (or c3 soup) inputs
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    w = torch.empty(nq, dtype=torch.float64, device="cuda")
    for _ in range(2):
        if args.case == "fp64_c3":
            rc = handle.wn_forward_fp64_device(tri.data_ptr(), ld, Ot.data_ptr(), w.data_ptr(),
                                               nf, nq, 0, sp)
        elif args.case == "closest_c3":
            tree = distance.DeviceAABB(V, F)
            w = tree.query(Ot)[0]
            tree.close()
            rc = 0
        elif args.case == "fwn_c3":
            import igl

            fwn = igl.FastWindingNumber(V, F)
            w = fwn.evaluate_torch(Ot, beta=2.0)
            torch.cuda.synchronize()
            fwn.close()
            rc = 0
        else:
            mesh = wa.PreparedMesh(tri, ld, nf)
            if args.case == "fp64_tiled_c3":
                rc = handle.wn_forward_fp64_mesh_device(mesh.mesh, Ot.data_ptr(), nq,
                                                        w.data_ptr(), sp)
            elif args.case == "mixed_c3":
                w = mesh.forward(Ot)
                rc = 0
            else:
                g = torch.from_numpy(np.random.default_rng(5).normal(size=nq)).cuda()
                w = mesh.backward(Ot, g)[0]
                rc = 0
            torch.cuda.synchronize()
            mesh.close()
        if rc != 0:
            raise RuntimeError(_lib.last_error(handle))
    torch.cuda.synchronize()
    if handle.wn_stream_check(sp) != 0:
        raise RuntimeError(_lib.last_error(handle))
    print("ok", args.case, nf, nq, float(w.double().abs().sum()))


def main():
    args = parse_args()
    if args.case:
        run_case(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
