#!/usr/bin/env python3
"""Benchmark of the k-d tree hot path on B200.

Workload (one step, per GPU): the 10M-point Gaussian-mixture configuration
-- 64 components, centres U[0,1)^3 (seed 3), sigma 0.01, stored as
{float3 p; uint32 payload} 16-byte records whose top two payload bits hold
the split dimension (widest extent of each node's domain) -- is built into a
left-balanced k-d tree in place, then k=16 nearest neighbours are found for
10M queries drawn from the same mixture (seed 4) with the stack-based
traversal.  value = queries answered per second with the build included in
every step (the step restores the unbuilt points first; inputs exceed the
126 MB L2, so no flush is needed between steps).

Run:  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Under torchrun each rank runs one replica on its own GPU (weak scaling:
queries and trees are independent, there is no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 10_000_000
N_QUERIES = 10_000_000
K = 16
RECORD_BYTES = 16
METRIC = "knn_queries_per_s"
UNIT = "queries/s"
WORKLOAD = ("build (widest-dim, 16-byte {float3,payload+dim} records) + kNN k=16 "
            "stack-based over 10M Gaussian-mixture points and 10M mixture queries")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=N_POINTS)
    ap.add_argument("--queries", type=int, default=N_QUERIES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(n_points, n_queries):
    from cudakdtree_b200 import workloads as wl
    pts = wl.gmm_points(n_points, seed=3)
    q = wl.gmm_points(n_queries, seed=3, sample_seed=4)
    return wl.packed_records(pts), q


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


def profile_traffic(key):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(key)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def max_over_ranks(t_ms, pg, device):
    """The slowest rank's device time (every rank takes the same collective)."""
    if not pg:
        return float(t_ms)
    import torch
    t = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_per_step):
    """Units all ranks processed per second (weak scaling: fixed work per rank)."""
    return world * units_per_rank / (ms_per_step / 1e3)


def run_ours(args, rank, world, local):
    import torch
    import cudakdtree_b200 as ck

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    recs, q = workload(args.points, args.queries)
    n, nq = len(recs), len(q)
    lay = ck.layout_for("float32", 3, stride=RECORD_BYTES, dim_offset=12, dim_shift=30,
                        dim_bits=2)
    h_pts = torch.from_numpy(recs.view(np.int32).reshape(n, 4).copy()).pin_memory()
    h_q = torch.from_numpy(q).pin_memory()
    d_src = h_pts.to(dev)
    d_pts = torch.empty_like(d_src)
    d_q = h_q.to(dev)
    d_ids = torch.empty((nq, K), dtype=torch.int32, device=dev)
    d_d2 = torch.empty((nq, K), dtype=torch.float32, device=dev)
    wb = torch.empty((2, 3), dtype=torch.float32, device=dev)

    def step():
        d_pts.copy_(d_src, non_blocking=True)
        ck.build_tree(d_pts, layout=lay, world_bounds=wb)
        ck.knn(d_pts, d_q, K, "stack_based", layout=lay, world_bounds=wb, out_ids=d_ids,
               out_d2=d_d2)

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = ck.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    barrier()
    launches = ck.launch_count() - l0
    clocks = sampler.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1), pg, dev)
    ms_per_step = t_ms / args.steps
    value = whole_job_rate(nq, world, ms_per_step)

    # ---- phase timings (same stream, CUDA events), outside the timed region
    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    def build_only():
        d_pts.copy_(d_src, non_blocking=True)
        ck.build_tree(d_pts, layout=lay, world_bounds=wb)

    copy_ms = timed(lambda: d_pts.copy_(d_src, non_blocking=True))
    build_ms = timed(build_only) - copy_ms
    # d_pts now holds the built tree
    knn_sb_ms = timed(lambda: ck.knn(d_pts, d_q, K, "stack_based", layout=lay, world_bounds=wb,
                                     out_ids=d_ids, out_d2=d_d2))
    knn_sf_ms = timed(lambda: ck.knn(d_pts, d_q, K, "stack_free", layout=lay, world_bounds=wb,
                                     out_ids=d_ids, out_d2=d_d2))
    knn_ref_ms = timed(lambda: ck.knn(d_pts, d_q, K, "stack_based", layout=lay,
                                      world_bounds=wb, out_ids=d_ids, out_d2=d_d2,
                                      reference_order=True), reps=1)
    morton_ms = timed(lambda: ck.morton_order(d_q))
    fcp_ms = timed(lambda: ck.fcp(d_pts, d_q, "stack_based", layout=lay, world_bounds=wb))

    # ---- learned radius vs plain on the same queries (config 4's method on
    # this workload: trained on 1M queries from the query distribution)
    learned = None
    if not args.no_learned:
        from cudakdtree_b200 import workloads as wl
        ntrain = min(1_000_000, nq)
        qtrain = torch.from_numpy(wl.gmm_points(ntrain, seed=3, sample_seed=14)).to(dev)
        model = ck.RadiusModel(grid_res=64, seed=1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        model.fit(d_pts, qtrain, K, layout=lay, world_bounds=wb, epochs=10, batch=4096)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        fb = [None]

        def run_learned():
            fb[0] = ck.knn_learned(d_pts, d_q, K, model, "stack_based", layout=lay,
                                   world_bounds=wb, scale=1.2, out_ids=d_ids, out_d2=d_d2)[2]

        learned_ms = timed(run_learned)
        learned = {"knn_ms": round(learned_ms, 3), "plain_knn_ms": round(knn_sb_ms, 3),
                   "speedup_vs_plain": round(knn_sb_ms / learned_ms, 3),
                   "reference_order_knn_ms": round(knn_ref_ms, 3),
                   "speedup_vs_reference_order": round(knn_ref_ms / learned_ms, 3),
                   "queries_per_s": round(nq / (learned_ms / 1e3), 1),
                   "fallback_rate": round(int(fb[0][0].item()) / nq, 5),
                   "reference_order_reruns": int(fb[0][1].item()),
                   "train_s": round(train_s, 3), "train_queries": ntrain,
                   "final_loss": round(model.final_loss, 5), "radius_scale": 1.2}

    # ---- roofline of the dominant kernel (kNN traversal)
    peak, peak_src = measured_peaks()
    visits = ck.knn_visits(d_pts, d_q, K, "stack_based", layout=lay, world_bounds=wb)
    tot_visits = int(visits.sum().item())
    knn_bytes = tot_visits * RECORD_BYTES + nq * 12 + nq * K * 8
    achieved = knn_bytes / (knn_sb_ms / 1e3) / 1e9
    traffic = profile_traffic("knn_stack_based_k16_10M")
    roofline = {"bound": "hbm", "kernel": "knn stack-based k=16 (cukd_knn: Morton order + "
                "query_kernel)", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "algorithmic_bytes": knn_bytes,
                "bytes_formula": "sum(visits_ref)*16 + nq*12 + nq*k*8",
                "mean_visits_per_query": round(tot_visits / nq, 2), "peak_source": peak_src}
    levels = int(math.floor(math.log2(n))) + 1
    build_bytes = 2 * n * RECORD_BYTES * levels
    build_roof = {"bound": "hbm", "achieved": round(build_bytes / (build_ms / 1e3) / 1e9, 1),
                  "peak": peak, "unit": "GB/s",
                  "frac": round(build_bytes / (build_ms / 1e3) / 1e9 / peak, 4),
                  "algorithmic_bytes": build_bytes, "bytes_formula": "2*N*16*L",
                  "traffic": profile_traffic("build_10M")}

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        h_ids = torch.empty((nq, K), dtype=torch.int32).pin_memory()
        h_d2 = torch.empty((nq, K), dtype=torch.float32).pin_memory()

        def e2e_step():
            d_pts.copy_(h_pts, non_blocking=True)
            d_q.copy_(h_q, non_blocking=True)
            ck.build_tree(d_pts, layout=lay, world_bounds=wb)
            ck.knn(d_pts, d_q, K, "stack_based", layout=lay, world_bounds=wb, out_ids=d_ids,
                   out_d2=d_d2)
            h_ids.copy_(d_ids, non_blocking=True)
            h_d2.copy_(d_d2, non_blocking=True)

        for _ in range(2):
            e2e_step()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            e2e_step()
        b.record()
        barrier()
        et = max_over_ranks(a.elapsed_time(b), pg, dev)
        e2e = {"value": round(whole_job_rate(nq, world, et / args.steps), 1), "unit": UNIT,
               "h2d_bytes_per_step": int(h_pts.numel() * 4 + h_q.numel() * 4),
               "d2h_bytes_per_step": int(h_ids.numel() * 4 + h_d2.numel() * 4),
               "ms_per_step": round(et / args.steps, 3)}

    batched = None if args.no_batched else batched_section(ck, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(d_pts.cpu().numpy(), wb.cpu().numpy(), q)

    out = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded Gaussian mixture, 64 components, sigma 0.01)",
           "config": {"workload": WORKLOAD, "points": n, "queries": nq, "k": K,
                      "record_bytes": RECORD_BYTES, "split": "widest extent (explicit dim)",
                      "traversal": "stack_based", "morton_reorder": True,
                      "l2": "inputs exceed L2 (160 MB points + 120 MB queries), no flush",
                      "parallelism": f"replicas x{world}"},
           "phases_ms": {"build": round(build_ms, 3), "knn_stack_based": round(knn_sb_ms, 3),
                         "knn_stack_free": round(knn_sf_ms, 3), "morton_order": round(morton_ms, 3),
                         "fcp_stack_based": round(fcp_ms, 3), "restore_copy": round(copy_ms, 3),
                         "knn_stack_based_reference_order": round(knn_ref_ms, 3)},
           "build_ms": round(build_ms, 3),
           "knn_stack_free_queries_per_s": round(nq / (knn_sf_ms / 1e3), 1),
           "learned_radius": learned, "batched": batched,
           "roofline": roofline, "build_roofline": build_roof,
           "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "gpu_launches": int(launches),
           "gpu_launches_per_step": round(launches / args.steps, 1)}
    if pg:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def batched_section(ck, dev):
    """Many clouds built and queried together (cukd_batch_*): 4096 clouds of
    floor(exp(U[ln 256, ln 65536])) uniform points, 1024 uniform queries
    each, k = 8, stack-based; autotuned, then timed as CUDA-graph replays
    of build + query (the input cloud array is restored before each)."""
    import torch
    from cudakdtree_b200 import workloads as wl
    pts, poff, qs, qoff = wl.batched_clouds()
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    src = torch.from_numpy(pts).to(dev)
    P = torch.empty_like(src)
    Q = torch.from_numpy(qs).to(dev)
    bnd = plan.bounds_tensor(dev)
    out = plan._outputs(dev)
    tune = plan.autotune(src, Q, reps=3)

    def run():
        P.copy_(src, non_blocking=True)
        plan.run(P, Q, bnd, out=out)

    def timed(fn, reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    copy_ms = timed(lambda: P.copy_(src, non_blocking=True), 5)
    l0 = ck.launch_count()
    run_ms = timed(run, 10) - copy_ms
    launches = (ck.launch_count() - l0) / 10
    P.copy_(src)
    build_ms = timed(lambda: (P.copy_(src, non_blocking=True), plan.build(P, bnd)), 5) - copy_ms
    query_ms = timed(lambda: plan.query(P, Q, bnd, out=out), 5)
    nq, n = qs.shape[0], pts.shape[0]
    del plan
    return {"workload": "4096 clouds, sizes floor(exp(U[ln 256, ln 65536])) (seed 5), uniform "
                        "points and 1024 uniform queries per cloud, float3, k=8, stack_based",
            "clouds": int(poff.size - 1), "points": int(n), "queries": int(nq), "k": 8,
            "tuning": {k: (round(v, 3) if isinstance(v, float) else v)
                       for k, v in tune.as_dict().items()},
            "run_ms": round(run_ms, 3), "build_ms": round(build_ms, 3),
            "query_ms": round(query_ms, 3),
            "queries_per_s": round(nq / (run_ms / 1e3), 1),
            "build_points_per_s": round(n / (build_ms / 1e3), 1),
            "kernel_launches_per_run": launches, "graph": True}


def cpu_baseline_sample(tree_records_i32, bounds, q):
    """The reference's own host code (oracle/_ref) on a bounded sample of
    the workload, on this box's host cores."""
    try:
        from oracle import pyoracle as po
        if po.ref_host() is None:
            return {"value": None, "unit": UNIT, "unavailable": "oracle/_ref not built"}
        from cudakdtree_b200 import workloads as wl
        cores = po.nthreads()
        rec = tree_records_i32.view(po.ref_record_dtype(po.REF_F3_PACKED)).reshape(-1)
        ns = min(len(q), 1_000_000)
        qs = np.ascontiguousarray(q[:ns])
        t = time.perf_counter()
        po.ref_knn_host(po.REF_F3_PACKED, rec, bounds, qs, K, po.STACK_BASED, threads=cores)
        tq = time.perf_counter() - t
        nb = 1_000_000
        sub = wl.packed_records(wl.gmm_points(nb, seed=3))
        sub_rec = sub.view(po.ref_record_dtype(po.REF_F3_PACKED))
        t = time.perf_counter()
        po.ref_build_host(po.REF_F3_PACKED, sub_rec)
        tb = time.perf_counter() - t
        return {"value": round(ns / tq, 1), "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": (f"reference stackBased::knn<FixedCandidateList<16>> (OpenMP, {cores} "
                           f"threads) on {ns} of the 10M queries against the full 10M-point tree "
                           "(query phase only; the tree is the GPU build, byte-identical to "
                           "buildTree_host's); reference buildTree_host on a 1M-point sample of "
                           f"the mixture took {tb:.2f} s single-threaded"),
                "build_1M_sample_s": round(tb, 3)}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "unavailable": repr(e)[:200]}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU implementation of the path
# ---------------------------------------------------------------------------
def run_reference(args, rank, world, local):
    if rank != 0:
        return
    from oracle import pyoracle as po
    if po.ref_host() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    recs, q = workload(args.points, args.queries)
    n, nq = len(recs), len(q)
    cores = po.nthreads()
    rec = recs.view(po.ref_record_dtype(po.REF_F3_PACKED))
    t = time.perf_counter()
    tree, bounds = po.ref_build_host(po.REF_F3_PACKED, rec)
    t_build = time.perf_counter() - t
    sample = min(nq, 1_000_000)

    def knn_sample(i):
        lo = (i * sample) % max(1, nq - sample + 1)
        qs = np.ascontiguousarray(q[lo:lo + sample])
        t0 = time.perf_counter()
        po.ref_knn_host(po.REF_F3_PACKED, tree, bounds, qs, K, po.STACK_BASED, threads=cores)
        return time.perf_counter() - t0

    for i in range(args.warmup):
        knn_sample(i)
    times = [knn_sample(args.warmup + i) for i in range(args.steps)]
    t_knn = float(np.mean(times)) * (nq / sample)
    step_s = t_build + t_knn
    value = nq / step_s
    desc = (f"cukd::buildTree_host (single-threaded, as the reference implements it) on all "
            f"{n} points timed once ({t_build:.2f} s) + stackBased::knn<FixedCandidateList<16>> "
            f"on {sample}-query samples per step with {cores} OpenMP threads, scaled to {nq} "
            "queries")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(step_s * 1e3, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (same seeds as our arm)",
           "config": {"workload": WORKLOAD, "points": n, "queries": nq, "k": K,
                      "parallelism": "host cores"},
           "build_ms": round(t_build * 1e3, 1),
           "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores,
                            "kind": "reference", "sample": desc},
           "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
