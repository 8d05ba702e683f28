"""Benchmark: output triangles/s of constrained-Delaunay quality refinement.

Workload (default): the large clustered configuration - 2,000,000 FP64 points
from 64 isotropic Gaussians (centres uniform in [0,1e4]^2, sigma log-uniform in
[5,200]) plus 10% uniform background, 100,000 non-crossing endpoint-disjoint
segments, CDT with the convex hull enclosed; theta = 20 deg, Ruppert mode,
Offcenter policy.  Inputs are synthetic and seeded (no dataset exists for it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is output triangles per second of the
refinement with the input CDT already resident in HBM; `e2e` is the same
metric through the reference-facing C ABI call (host arrays in, host arrays
out, copies included).  The working set (input CDT ~130 MB plus the mesh
arrays) exceeds the 126 MB L2, so no explicit flush is done between steps.

--impl reference times the reference's own CPU quality refinement (Triangle
1.6 as vendored by the reference, triangulate("pzDQnrq20"),
GPU_Refine/main.cpp:389-407) compiled from the reference sources into
oracle/_ref, on the full workload and on all host cores: Triangle refines one
mesh on one thread, so every step is one full refinement in a process of its
own, as many at a time as there are cores; value = output triangles of all
timed steps / the wall time of the timed steps.

Multi-GPU: the single-domain refinement does not shard (its rounds resolve
conflicts globally), so --gpus N runs N independent replicas, one per GPU,
each refining the full workload; value is the sum over ranks of output
triangles divided by the slowest rank's time ("scaling": "weak").  The
batched workload shards by domain: with N > 1 the line also carries the
4,096-domain batch distributed over the ranks (replicas.refine_batch_sharded,
no data-path collective), timed as the slowest rank's engine call.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "output triangles/s at theta=20 deg, 1 B200 (learned vs plain); output vertex count"

# Algorithmic bytes of the flip-step check kernel (k_check_flip2, the
# kernelCheckFlipping of GPU_Refine/refine.cu:778-1070) per active triangle:
# the list entry (4), the triangle's vertices, neighbours and subsegments
# (3 x 12), the redundant flags of its vertices (3), its three points (48),
# per edge the neighbour's flip flag, opposite vertex, its flag and point
# (3 x 22), and the deferred-clear byte written back (1).
CHECK_BYTES_PER_ITEM = 4 + 36 + 3 + 48 + 66 + 1
# DRAM bytes (read + write) per active triangle of the same kernel, from
# `ncu --set full` on its first launch of the 1,000,000-point clustered case
# (profiles/k_check_flip2_clustered1M.md: 72.22 MB for 162,684 triangles).
CHECK_DRAM_BYTES_PER_ITEM = 72.22e6 / 162684
# FP64-pipe utilisation of the same launch (sm__inst_executed_pipe_fp64, % of
# peak sustained active): the exact-predicate filters are a small part of its work.
CHECK_FP64_PIPE_PCT = 4.26
# Algorithmic bytes of one whole flip step, for the small-step kernel (it runs
# every phase of a step in one launch), per active triangle: the check
# (CHECK_BYTES_PER_ITEM), the winner test (list entry 4, deferred-clear byte
# 1, flip orientation 1, the claim words of the triangle and its partner 8)
# and the filter into the next active set (queue entry 4, flip flag 1, status
# 1, list entry written 4) ...
STEP_BYTES_PER_ITEM = CHECK_BYTES_PER_ITEM + 14 + 10
# ... and per flip or flop applied: the vertex, neighbour and subsegment rows
# (48 B) of its two triangles read and written, and the back pointers of their
# four outer neighbours read and written (4 x 8).
STEP_BYTES_PER_WINNER = 2 * 2 * 48 + 4 * 8


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--points", type=int, default=2_000_000)
    p.add_argument("--segments", type=int, default=100_000)
    p.add_argument("--seed", type=int, default=20261205)
    p.add_argument("--cpu-baseline", type=int, default=1, help="time the CPU baseline (rank 0, N=1)")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--batch-domains", type=int, default=4096,
                   help="also time the batched workload with this many domains (0: skip)")
    p.add_argument("--batch-sample", type=int, default=64,
                   help="domains refined one call each to time the per-domain path")
    p.add_argument("--extras", type=int, default=1,
                   help="also measure the adversarial input and the learned placement (0: skip)")
    p.add_argument("--autotune", type=int, default=1,
                   help="choose the flip-loop launch shape with the autotuner before timing (0: defaults)")
    return p.parse_args()


def workload(args):
    """The clustered input of inputs.clustered, keeping its points and segments."""
    from gpu_cdt_refine_b200 import inputs
    t0 = time.time()
    pts = inputs.cluster_points(args.points, 64, 1.0e4, 5.0, 200.0, 0.10, args.seed)
    seg = inputs.pick_segments(pts, args.segments, args.seed + 1)
    cdt = inputs.build_cdt(pts, seg)
    return cdt, time.time() - t0, pts, seg


def config(args, cdt):
    return {"workload": "clustered Gaussian mixture, theta=20 Ruppert Offcenter",
            "points_in": cdt.numberofpoints, "triangles_in": cdt.numberoftriangles,
            "segments_in": cdt.numberofsegments, "theta": 20.0, "mode": "ruppert", "policy": "offcenter",
            "predicates": "reference", "l2": "working set larger than L2 (126 MB); no flush",
            "seed": args.seed}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for k, n in enumerate(names):
                    if s[5 + k].lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    """The host CPU's model name and logical core count, reported beside every CPU baseline."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical cores"


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_batch_workload(args, local_rank):
    """The batched workload (independent domains, N log-uniform in [200, 50000],
    uniform or 1-8 Gaussian clusters, segments 5% of N, theta from {15, 18, 20},
    Ruppert, Offcenter) through the persistent engine, against single-domain
    calls on a seeded sample of the same domains (time scaled to all domains)."""
    from gpu_cdt_refine_b200 import inputs, refine
    t0 = time.time()
    doms, thetas = inputs.batch_domains(args.batch_domains)
    gen_s = time.time() - t0
    rng = np.random.default_rng(7)
    n = len(doms)
    tune = sorted(rng.choice(n, min(256, n), replace=False).tolist())
    chosen, tune_ms = refine.batch_autotune([doms[i] for i in tune], [thetas[i] for i in tune], device=local_rank)
    refine.refine_batch_persistent(doms, thetas, device=local_rank)  # warm-up (buffers grow once)
    t0 = time.perf_counter()
    got, _, rep = refine.refine_batch_persistent(doms, thetas, device=local_rank, with_report=True)
    call_ms = (time.perf_counter() - t0) * 1e3
    tris = sum(g.numberoftriangles for g in got)
    samp = sorted(rng.choice(n, min(args.batch_sample, n), replace=False).tolist())
    refine.refine(doms[samp[0]], thetas[samp[0]], device=local_rank)
    t0 = time.perf_counter()
    for i in samp:
        refine.refine(doms[i], thetas[i], device=local_rank)
    single_ms = (time.perf_counter() - t0) * 1e3 * n / len(samp)
    try:
        cpu = batch_cpu_baseline(doms, thetas) if args.cpu_baseline else None
    except Exception as e:  # the reference build is test infrastructure; report, do not fail
        cpu = {"value": None, "unit": "triangles/s", "kind": "reference", "sample": f"unavailable: {e}"}
    return {"workload": f"{n} independent domains, N log-uniform [200, 50000], uniform or 1-8 Gaussian clusters, "
                        f"segments 5% of N, theta in {{15, 18, 20}}, Ruppert, Offcenter",
            "domains": n, "points_in": int(sum(d.numberofpoints for d in doms)), "output_triangles": int(tris),
            "kernel_ms": rep["kernel_ms"], "call_ms": call_ms, "report": rep,
            "triangles_per_s_call": tris / (call_ms / 1e3), "triangles_per_s_kernel": tris / (rep["kernel_ms"] / 1e3),
            "variant": list(chosen), "autotune_ms": {f"{k[0]}x{k[1]}": v for k, v in tune_ms.items()},
            "per_domain_calls_ms": single_ms,
            "per_domain_sample": f"{len(samp)} seeded domains, one gqm_refine call each (host arrays in and out), "
                                 f"time scaled by {n}/{len(samp)}",
            "cpu_baseline": cpu, "generation_s": gen_s}


def _triangle_worker(ids, seed, barrier, out):
    """One host core of the batch's CPU baseline: builds its domains (untimed),
    waits for the other workers, then refines its domains one after another
    with Triangle -q and reports (output triangles, seconds).  Triangle keeps
    its state in globals, so each core is a process of its own."""
    from gpu_cdt_refine_b200 import inputs
    from oracle import tri_ref
    work = [inputs.batch_domain(seed + 2 * k) for k in ids]
    barrier.wait(timeout=300)
    t0 = time.perf_counter()
    tris = 0
    for cdt, theta in work:
        tris += tri_ref.quality(cdt, theta, 1)[1]
    out.put((tris, time.perf_counter() - t0, sum(c.numberofpoints for c, _ in work)))


def batch_cpu_baseline(doms, thetas, seed=20261207):
    """Triangle's quality refinement (pzDQnrq<theta>, the reference's CPU path)
    of every domain of the batch on all host cores: one spawned process per
    core (no CUDA state is inherited), domains assigned by the same
    cost-balanced partition as the multi-GPU batch, all workers released
    together; triangles/s = output triangles / the slowest worker's time."""
    import multiprocessing as mp
    from gpu_cdt_refine_b200 import replicas
    cores = max(1, min(os.cpu_count() or 1, len(doms)))
    parts, _ = replicas.partition_domains([replicas.domain_cost(d.numberofpoints, t) for d, t in zip(doms, thetas)],
                                          cores)
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(cores), ctx.Queue()
    procs = [ctx.Process(target=_triangle_worker, args=(p, seed, barrier, out), daemon=True) for p in parts]
    for p in procs:
        p.start()
    try:
        res = [out.get(timeout=600) for _ in procs]
    finally:  # a worker that failed leaves no process behind
        for p in procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()
    tris, wall = sum(r[0] for r in res), max(r[1] for r in res)
    if sum(r[2] for r in res) != sum(d.numberofpoints for d in doms):
        raise RuntimeError("the workers' domains differ from the batch")
    return {"value": tris / wall, "unit": "triangles/s", "cores": cores, "kind": "reference", "host": cpu_model(),
            "sample": f"Triangle 1.6 pzDQnrq<theta> on all {len(doms)} domains of the batch, one process per core, "
                      f"{wall:.1f} s wall (slowest core), {sum(r[1] for r in res):.1f} s of CPU work",
            "output_triangles": int(tris), "wall_ms": wall * 1e3}


def run_adversarial(local_rank):
    """The adversarial input (1,000,000 points: a 700 x 700 grid jittered by
    1e-9 of its spacing plus 200 concentric circles, 20,000 chords along the
    circles), theta 20.7, Ruppert, Offcenter, with the reference's predicate
    arithmetic and with exact predicates; incircle tests that needed the
    expansion path are counted on the device."""
    from gpu_cdt_refine_b200 import inputs, refine
    from gpu_cdt_refine_b200.certify import certify
    t0 = time.time()
    cdt = inputs.adversarial()
    gen_s = time.time() - t0
    out = {"workload": "700x700 jittered grid + 200 concentric circles, 20,000 chords, theta 20.7, Ruppert, "
                       "Offcenter", "points_in": cdt.numberofpoints, "segments_in": cdt.numberofsegments,
           "generation_s": gen_s}
    for name, pred in (("reference_predicates", refine.PRED_REFERENCE), ("exact_predicates", refine.PRED_EXACT)):
        refine.refine(cdt, 20.7, refine.Offcenter, 1, predicates=pred, device=local_rank)
        got, st = refine.refine(cdt, 20.7, refine.Offcenter, 1, predicates=pred, device=local_rank)
        cert = certify(got, cdt, 20.7)
        out[name] = {"device_ms": st["device_ms"], "output_triangles": got.numberoftriangles,
                     "output_vertices": got.numberofpoints, "incircle_expansion_fallbacks": st["exact_fallbacks"],
                     "fallbacks_per_output_triangle": st["exact_fallbacks"] / max(got.numberoftriangles, 1),
                     "certified": bool(cert["ok"]), "min_angle_deg": cert["min_angle_deg"],
                     "triangles_below_theta": cert["triangles_below_theta"]}
    return out


def run_learned(cdt, args, local_rank):
    """Learned Steiner placement (the network trained by train_placement.py,
    gpu_cdt_refine_b200/data/placement_mlp.npy) against the plain rule: the
    clustered input of the main workload and 256 batched domains."""
    from gpu_cdt_refine_b200 import inputs, refine
    from gpu_cdt_refine_b200.certify import certify
    path = os.path.join(ROOT, "gpu_cdt_refine_b200", "data", "placement_mlp.npy")
    params = np.load(path).astype(np.float32)
    res = {"network": "gpu_cdt_refine_b200/data/placement_mlp.npy (descendant-count labels: exploration runs of 128 "
                      "seeded clustered inputs of 200,000 points, theta 20, 33 levels of t, 5 generations, 4 "
                      "regression networks averaged)"}
    plain, sp = refine.refine(cdt, 20.0, refine.Offcenter, 1, device=local_rank)
    learned, sl = refine.refine(cdt, 20.0, refine.Offcenter, 1, device=local_rank, mlp=params)
    learned, sl = refine.refine(cdt, 20.0, refine.Offcenter, 1, device=local_rank, mlp=params)
    cert = certify(learned, cdt, 20.0)
    res["clustered_2M"] = {"plain_vertices": plain.numberofpoints, "learned_vertices": learned.numberofpoints,
                           "vertex_reduction": 1.0 - learned.numberofpoints / plain.numberofpoints,
                           "plain_device_ms": sp["device_ms"], "learned_device_ms": sl["device_ms"],
                           "candidates": sl["learned_candidates"], "network_points": sl["learned_used"],
                           "fallback_rate": 1.0 - sl["learned_used"] / max(sl["learned_candidates"], 1),
                           "certified": bool(cert["ok"]), "min_angle_deg": cert["min_angle_deg"],
                           "triangles_below_theta": cert["triangles_below_theta"]}
    # the network alone: one inference launch over as many rows as the run had
    # candidates (the run spreads them over its rounds, with the features)
    mlp_ms = refine.mlp_time(params, sl["learned_candidates"], device=local_rank)
    res["clustered_2M"].update({"mlp_ms_all_candidates": mlp_ms, "mlp_share_of_learned_run": mlp_ms / sl["device_ms"]})
    doms, _ = inputs.batch_domains(256, seed=20261209)
    gp, _, rp = refine.refine_batch_persistent(doms, 20.0, device=local_rank, with_report=True)
    gl, stl, rl = refine.refine_batch_persistent(doms, 20.0, device=local_rank, with_report=True, mlp=params)
    pv, lv = sum(g.numberofpoints for g in gp), sum(g.numberofpoints for g in gl)
    cand, used = sum(s["learned_candidates"] for s in stl), sum(s["learned_used"] for s in stl)
    res["batch_256"] = {"plain_vertices": pv, "learned_vertices": lv, "vertex_reduction": 1.0 - lv / pv,
                        "plain_kernel_ms": rp["kernel_ms"], "learned_kernel_ms": rl["kernel_ms"],
                        "fallback_rate": 1.0 - used / max(cand, 1)}
    return res


def run_construction(pts, seg, e2e_ms, local_rank):
    """CDT construction, the step in front of the refiner: the GPU builder
    against the reference's own input builder (Triangle "pzQnc",
    GPU_Refine/mesh.cpp:397, one host core) and this repository's exact CPU
    builder on the same points and segments; then the whole flow from points
    and segments to the refined mesh in one device-resident call."""
    from gpu_cdt_refine_b200 import cdtio, inputs, triangulate
    res = {"workload": f"{pts.shape[0]} clustered points, {seg.shape[0]} segments (the input of the main workload)"}
    walls, st, g = [], None, None
    for i in range(4):
        t0 = time.perf_counter()
        g, st = triangulate.build_cdt_gpu(pts, seg, device=local_rank, with_stats=True)
        if i:
            walls.append((time.perf_counter() - t0) * 1e3)
    res["gpu_ms"] = float(np.median(walls))
    res["gpu_phases_ms"] = {k: st[k] for k in ("ms_h2d", "ms_hull", "ms_insert", "ms_segments", "ms_output", "ms_d2h")}
    res["gpu_counts"] = {k: st[k] for k in ("insert_rounds", "flip_rounds", "recover_rounds", "segments_missing",
                                            "flips", "recover_flips", "kernel_launches", "hull_vertices")}
    t0 = time.perf_counter()
    mine = inputs.build_cdt(pts, seg)
    res["cpu_builder_ms"] = (time.perf_counter() - t0) * 1e3
    res["same_as_cpu_builder"] = bool(cdtio.same_mesh(mine, g))
    try:
        from oracle import tri_ref
        tri, tri_ms = tri_ref.cdt(pts, seg, with_ms=True)
        res["triangle_ms"] = tri_ms
        res["triangle_cores"] = 1
        res["same_as_triangle"] = bool(cdtio.same_mesh(tri, g))
        res["speedup_vs_triangle"] = tri_ms / res["gpu_ms"]
    except Exception as e:  # the reference build is test infrastructure; report, do not fail
        res["triangle_ms"] = None
        res["triangle_unavailable"] = str(e)
    # the first call builds the contexts, the second allocates the second pinned
    # result block (the first result is still held): both are set-up, not steady state
    walls = []
    for i in range(5):
        t0 = time.perf_counter()
        out, _, _ = triangulate.triangulate_refine(pts, seg, device=local_rank)
        if i >= 2:
            walls.append((time.perf_counter() - t0) * 1e3)
    res["points_to_refined_mesh_ms"] = float(np.median(walls))
    res["points_to_refined_mesh_triangles"] = out.numberoftriangles
    if res.get("triangle_ms") is not None:
        res["triangle_cdt_then_refine_ms"] = res["triangle_ms"] + e2e_ms
    return res


def _triangle_step(path, theta, mode):
    """One step of the reference arm, in a spawned process: Triangle's quality
    refinement of the CDT stored at `path`; returns (ms, output triangles)."""
    from gpu_cdt_refine_b200 import cdtio
    from oracle import tri_ref
    return tri_ref.quality(cdtio.read_cdt(path), theta, mode)


def triangle_steps(cdt, count, workers, theta=20.0, mode=1):
    """`count` full Triangle refinements of `cdt`, `workers` processes at a
    time (spawned, so no CUDA state is inherited); returns (wall s, list of
    (ms, triangles))."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import tempfile
    from gpu_cdt_refine_b200 import cdtio
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "workload.bin")
        cdtio.write_cdt(path, cdt)
        with cf.ProcessPoolExecutor(max(1, min(workers, count)), mp_context=mp.get_context("spawn")) as ex:
            ex.submit(int, 0).result()  # processes up before the clock starts
            t0 = time.perf_counter()
            runs = list(ex.map(_triangle_step, [path] * count, [theta] * count, [mode] * count))
            wall = time.perf_counter() - t0
    return wall, runs


def run_reference(args, rank, world):
    """The reference's CPU quality refinement on the full workload, every host
    core used: one Triangle process per step, as many at a time as cores."""
    if rank != 0:
        return
    full = workload(args)[0]
    cores = os.cpu_count() or 1
    triangle_steps(full, args.warmup, cores)  # warm-up steps, untimed
    wall, runs = triangle_steps(full, args.steps, cores)
    tris = sum(r[1] for r in runs)
    value = tris / wall
    single = float(np.mean([r[1] / (r[0] / 1e3) for r in runs]))
    line = {"metric": METRIC, "value": value, "unit": "triangles/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "impl": "reference", "config": config(args, full),
            "cpu_baseline": {"value": value, "unit": "triangles/s", "cores": min(cores, args.steps),
                             "kind": "reference", "host": cpu_model(),
                             "sample": f"Triangle 1.6 pzDQnrq20 (as vendored by the reference; one refinement per "
                                       f"thread) on the full workload ({full.numberofpoints} points, "
                                       f"{full.numberofsegments} segments), {args.steps} timed refinements, "
                                       f"{min(cores, args.steps)} at a time in processes of their own; "
                                       f"{wall:.1f} s wall",
                             "single_refinement_ms": float(np.mean([r[0] for r in runs])),
                             "single_core_value": single},
            "e2e": {"value": value, "unit": "triangles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "output_triangles": int(runs[0][1])}
    print(json.dumps(line), flush=True)


def kernel_rooflines(probe, ms_step, peak, peak_kind):
    """Roofline entries of the two kernels that take most of the device time,
    from the per-launch device timers of one probed refinement: the grid-wide
    flip-step check kernel (CHECK_BYTES_PER_ITEM per active triangle) and the
    small-step kernel (STEP_BYTES_PER_ITEM per active triangle plus
    STEP_BYTES_PER_WINNER per flip applied, summed over the steps it ran)."""
    out = []
    launches = max(int(probe["check_launches"]), 1)
    if probe["check_ms"] > 0:
        items = probe["check_items"] / launches
        launch_s = probe["check_ms"] / 1e3 / launches
        ach = CHECK_BYTES_PER_ITEM * items / launch_s / 1e9
        out.append({"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "traffic": CHECK_DRAM_BYTES_PER_ITEM * items, "peak_kind": peak_kind,
                    "kernel": "k_check_flip2 (grid-wide flip-step check)", "bytes_per_item": CHECK_BYTES_PER_ITEM,
                    "launches": launches, "items_per_launch": items, "avg_launch_us": launch_s * 1e6,
                    "share_of_step": probe["check_ms"] / ms_step,
                    "traffic_note": "ncu DRAM bytes per active triangle of the 1M-point capture "
                                    "(profiles/k_check_flip2_clustered1M.md) times this launch's items",
                    "fp64_pipe_pct_ncu": CHECK_FP64_PIPE_PCT})
    sl = max(int(probe["small_launches"]), 1)
    if probe["small_ms"] > 0:
        alg = STEP_BYTES_PER_ITEM * probe["small_items"] + STEP_BYTES_PER_WINNER * probe["small_winners"]
        launch_s = probe["small_ms"] / 1e3 / sl
        ach = alg / sl / launch_s / 1e9
        out.append({"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "traffic": None, "peak_kind": peak_kind,
                    "kernel": "small-step kernel (whole flip steps of small active sets in one launch)",
                    "bytes_per_item": STEP_BYTES_PER_ITEM, "bytes_per_winner": STEP_BYTES_PER_WINNER,
                    "launches": sl, "items_per_launch": probe["small_items"] / sl,
                    "winners_per_launch": probe["small_winners"] / sl, "avg_launch_us": launch_s * 1e6,
                    "share_of_step": probe["small_ms"] / ms_step})
    out.sort(key=lambda r: -r["share_of_step"])
    return out


def run_sharded_batch(args, world, local_rank, dev):
    """The batched workload over all ranks: every rank builds the same domain
    list, replicas.refine_batch_sharded gives each rank its cost-balanced share
    and times its engine call; the job time is the slowest rank's."""
    from gpu_cdt_refine_b200 import inputs, refine, replicas
    doms, thetas = inputs.batch_domains(args.batch_domains)
    mine = replicas.partition_domains([replicas.domain_cost(d.numberofpoints, t) for d, t in zip(doms, thetas)],
                                      world)[0]
    import torch.distributed as dist
    own = mine[dist.get_rank()]
    if own:  # warm-up: this rank's buffers grow once
        refine.refine_batch_persistent([doms[i] for i in own], [thetas[i] for i in own], device=local_rank)
    dist.barrier()
    ids, res, _, rep = replicas.refine_batch_sharded(doms, thetas, gather=False, device=local_rank)
    tris_all = replicas.reduce_step(0.0, float(sum(r.numberoftriangles for r in res)), device=dev)[1]
    return {"workload": f"{len(doms)} independent domains (the batched workload) sharded over {world} ranks",
            "domains_per_rank": rep["domains"], "max_ms": rep["max_ms"], "rank0_ms": rep["rank_ms"],
            "output_triangles": int(tris_all), "value": tris_all / (rep["max_ms"] / 1e3), "unit": "triangles/s",
            "timing": "each rank's wall time of its engine call (pack, upload, one persistent launch, download, "
                      "unpack); max over ranks by all-reduce"}


def run_ours(args, rank, world, local_rank):
    import torch
    from gpu_cdt_refine_b200 import refine

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    cdt, gen_s, raw_pts, raw_seg = workload(args)
    # inputs resident in HBM
    d_pts = torch.from_numpy(cdt.pointlist).to(dev)
    d_tri = torch.from_numpy(cdt.trianglelist).to(dev)
    d_nbr = torch.from_numpy(cdt.neighborlist).to(dev)
    d_seg = torch.from_numpy(cdt.segmentlist).to(dev)
    torch.cuda.synchronize()
    ctx = refine.Context(local_rank)
    opt = refine.make_options(20.0, refine.Offcenter, 1, device=local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    # launch shape of the flip-flop loop chosen by the autotuner on this input
    # (untimed; no shape changes a result)
    t0 = time.perf_counter()
    tuned, tuned_ms = ctx.autotune(cdt, opt) if args.autotune else (ctx.tuning(), None)
    autotune_s = time.perf_counter() - t0

    def step():
        return ctx.run_device(cdt.numberofpoints, cdt.numberoftriangles, cdt.numberofsegments, d_pts.data_ptr(),
                              d_tri.data_ptr(), d_nbr.data_ptr(), d_seg.data_ptr(), opt)

    for _ in range(args.warmup):
        st = step()
    np_out, nt_out, ns_out = ctx.sizes()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with Clocks(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            stats.append(step())
        ev1.record(stream)
        torch.cuda.synchronize()
    ms_total = ev0.elapsed_time(ev1)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = ms_total / args.steps
    # one more step with the device-side launch timers of the two main kernels on
    ctx.probe(True)
    step()
    probe = ctx.probe_read()
    ctx.probe(False)
    from gpu_cdt_refine_b200 import replicas
    ms_max, tris_all = replicas.reduce_step(ms, nt_out, device=dev)
    value = tris_all / (ms_max / 1e3)

    # end to end through the reference-facing call: host arrays in, host arrays
    # out (the autotuned shape set on the library's cached context of this device)
    refine.set_default_tuning(local_rank, **{k: v for k, v in tuned.items()})
    e2e_ms, h2d, d2h = [], cdt.nbytes(), 0
    refine.refine(cdt, 20.0, refine.Offcenter, 1, device=local_rank)  # warm-up of the cached context
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        out, _ = refine.refine(cdt, 20.0, refine.Offcenter, 1, device=local_rank)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        d2h = out.nbytes() + out.numberofpoints + out.numberoftriangles
    e2e_max, _ = replicas.reduce_step(float(np.median(e2e_ms)), nt_out, device=dev)
    e2e_value = tris_all / (e2e_max / 1e3)
    sharded = run_sharded_batch(args, world, local_rank, dev) if (world > 1 and args.batch_domains > 0) else None

    if rank == 0:
        peak, peak_kind = measured_peak()
        s = stats[-1]
        roofs = kernel_rooflines(probe, ms, peak, peak_kind)
        # path-level algorithmic bytes (input + output mesh + one quality check of
        # every output triangle): 16 B/point, 24 B/triangle, 8 B/segment, 60 B/tri
        alg = (16 * cdt.numberofpoints + 24 * cdt.numberoftriangles + 8 * cdt.numberofsegments + 16 * np_out +
               24 * nt_out + 8 * ns_out + 60 * nt_out)
        path_gbs = alg / (ms / 1e3) / 1e9
        top = dict(roofs[0]) if roofs else {}
        top.update({"timing": "per-launch device timers (%globaltimer, first block start to last block end) in "
                              "one extra probed step after the timed region, on the context's stream",
                    "path_achieved_gbs": path_gbs, "path_frac": path_gbs / peak, "kernels": roofs})
        cfg = config(args, cdt)
        cfg["launch_shape"] = tuned
        line = {"metric": METRIC, "value": value, "unit": "triangles/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
                "config": cfg,
                "output_vertices": np_out, "output_triangles": nt_out, "output_segments": ns_out,
                "e2e": {"value": e2e_value, "unit": "triangles/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_max},
                # kernels of the timed region (the library counts the kernels run
                # inside its flip-loop graphs as well as the launches from the host)
                "gpu_launches": int(sum(x["kernel_launches"] for x in stats)),
                "gpu_launches_per_refinement": int(s["kernel_launches"]),
                "host_syncs": int(s["host_syncs"]), "rounds": int(s["rounds"]),
                "flip_steps": int(s["flip_steps"]), "device_ms_library": s["device_ms"],
                "autotune": {"chosen": tuned, "best_ms": tuned_ms, "seconds": autotune_s},
                "roofline": top, "clocks": clk.summary(), "input_generation_s": gen_s}
        if sharded:
            line["batch_sharded"] = sharded
        if world == 1:
            line["other_modes"] = run_other_modes(ctx, cdt, local_rank)
        if args.batch_domains > 0 and world == 1:
            line["batch"] = run_batch_workload(args, local_rank)
        if args.extras and world == 1:
            line["construction"] = run_construction(raw_pts, raw_seg, e2e_max, local_rank)
            line["learned"] = run_learned(cdt, args, local_rank)
            line["adversarial"] = run_adversarial(local_rank)
        if args.cpu_baseline and world == 1:
            try:
                wall, runs = triangle_steps(cdt, 1, 1)
                ms_cpu, ntc = runs[0]
                line["cpu_baseline"] = {"value": ntc / (ms_cpu / 1e3), "unit": "triangles/s", "cores": 1,
                                        "kind": "reference", "host": cpu_model(),
                                        "sample": f"Triangle 1.6 pzDQnrq20 on the full workload "
                                                  f"({cdt.numberofpoints} points, {cdt.numberofsegments} "
                                                  f"segments), one refinement on one core, {ms_cpu / 1e3:.1f} s",
                                        "output_triangles": int(ntc)}
            except Exception as e:  # the reference build is test infrastructure; report, do not fail
                line["cpu_baseline"] = {"value": None, "unit": "triangles/s", "cores": 1, "kind": "reference",
                                        "sample": f"unavailable: {e}"}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def run_other_modes(ctx, cdt, local_rank):
    """The same input in the other three {mode} x {policy} combinations of the
    workload's configuration: device time of one refinement after a warm-up."""
    from gpu_cdt_refine_b200 import refine
    out = {}
    for name, policy, mode in (("ruppert_circumcenter", refine.Circumcenter, 1), ("chew_offcenter", refine.Offcenter, 0),
                               ("chew_circumcenter", refine.Circumcenter, 0)):
        opt = refine.make_options(20.0, policy, mode, device=local_rank)
        ctx.run_host(cdt, opt)
        st = ctx.run_host(cdt, opt)
        npo, nto, _ = ctx.sizes()
        out[name] = {"device_ms": st["device_ms"], "output_triangles": nto, "output_vertices": npo,
                     "triangles_per_s_device": nto / (st["device_ms"] / 1e3), "rounds": st["rounds"]}
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
