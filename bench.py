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
PARITY_SAMPLE = 1_000_000
# the learned radius network's training loss: pinball at this quantile of the
# k-th distance (fewer fallbacks than the mean-squared-error fit at the same
# radius scale, measured on the 10M-point benchmark and on config 4)
LEARNED_QUANTILE = 0.9
UNIT = "queries/s"


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
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the C1 / C4 / C5 measurements of the default line")
    ap.add_argument("--kernel-case", default="", choices=[""] + sorted(KERNEL_CASES),
                    help="run one small single-kernel case twice (the workloads of the "
                         "per-kernel ncu captures summarised under profiles/) and exit")
    ap.add_argument("--batched-clouds", type=int, default=4096,
                    help="clouds in the batched section (4096 = the configuration)")
    ap.add_argument("--batched-tuning", default="",
                    help="tile,block,queries_per_thread,morton for the batched section "
                         "instead of autotuning (profiling runs)")
    ap.add_argument("--e2e-chunk", type=int, default=1 << 21,
                    help="queries per chunk of the host-buffer kNN in the e2e measurements "
                         "that run one step at a time")
    ap.add_argument("--e2e-async-chunk", type=int, default=0,
                    help="queries per chunk of the pipelined e2e steps (0 = the library's "
                         "default for the asynchronous calls: the whole 10M batch)")
    ap.add_argument("--configs", default="",
                    help="comma list of c1,c2,c4,c5: measure those configurations instead "
                         "(one JSON line each, not the benchmark line)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_desc(n, nq):
    def m(x):
        return f"{x / 1e6:g}M" if x >= 1e6 else str(x)
    return (f"build (widest-dim, 16-byte {{float3,payload+dim}} records) + kNN k={K} "
            f"stack-based over {m(n)} Gaussian-mixture points and {m(nq)} mixture queries")


def bench_config(n, nq, world):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": workload_desc(n, nq), "points": n, "queries": nq, "k": K,
            "record_bytes": RECORD_BYTES, "split": "widest extent (explicit dim)",
            "traversal": "stack_based", "morton_reorder": True,
            "l2": "inputs exceed L2 (160 MB points + 120 MB queries), no flush",
            "parallelism": f"replicas x{world}"}


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
    # the last step's answers for the first PARITY_SAMPLE queries: checked
    # against the reference's host traversal in the CPU-baseline leg
    ns = min(nq, PARITY_SAMPLE)
    step_out = (d_ids[:ns].cpu().numpy(), d_d2[:ns].cpu().numpy())

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
    # the traversal kernel without the reorder: the same queries already in
    # Morton order (cukd_knn then runs knn_fast_kernel and the re-run of the
    # few tied queries)
    d_qs = d_q[ck.morton_order(d_q).long()].contiguous()
    knn_kernel_ms = timed(lambda: ck.knn(d_pts, d_qs, K, "stack_based", layout=lay,
                                         world_bounds=wb, out_ids=d_ids, out_d2=d_d2,
                                         morton=False))
    del d_qs
    fcp_ms = timed(lambda: ck.fcp(d_pts, d_q, "stack_based", layout=lay, world_bounds=wb))

    # ---- learned radius vs plain on the same queries (config 4's method on
    # this workload: trained on 1M queries from the query distribution)
    learned = None
    learned_out = None
    if not args.no_learned:
        from cudakdtree_b200 import workloads as wl
        ntrain = min(1_000_000, nq)
        qtrain = torch.from_numpy(wl.gmm_points(ntrain, seed=3, sample_seed=14)).to(dev)
        model = ck.RadiusModel(grid_res=64, seed=1, quantile=LEARNED_QUANTILE)
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
        learned_out = (d_ids[:ns].cpu().numpy(), d_d2[:ns].cpu().numpy())
        learned = {"knn_ms": round(learned_ms, 3), "plain_knn_ms": round(knn_sb_ms, 3),
                   "speedup_vs_plain": round(knn_sb_ms / learned_ms, 3),
                   "target_speedup_vs_plain": 1.5,
                   "target_met": bool(knn_sb_ms / learned_ms >= 1.5),
                   "path": ("cukd_knn_learned: Morton order, knn_learned_kernel (MLP on the "
                            "tensor cores fused with the seeded traversal), plain re-run of "
                            "the fallbacks, reference-order re-run of ties"),
                   "queries_per_s": round(nq / (learned_ms / 1e3), 1),
                   "fallback_rate": round(int(fb[0][0].item()) / nq, 5),
                   "reference_order_reruns": int(fb[0][1].item()),
                   "train_s": round(train_s, 3), "train_queries": ntrain,
                   "training_loss": f"pinball at quantile {LEARNED_QUANTILE}",
                   "final_loss": round(model.final_loss, 5), "radius_scale": 1.2}

    # ---- roofline of the dominant kernel (kNN traversal)
    peak, peak_src = measured_peaks()
    visits = ck.knn_visits(d_pts, d_q, K, "stack_based", layout=lay, world_bounds=wb)
    tot_visits = int(visits.sum().item())
    knn_bytes = tot_visits * RECORD_BYTES + nq * 12 + nq * K * 8
    achieved = knn_bytes / (knn_kernel_ms / 1e3) / 1e9
    traffic = profile_traffic("knn_stack_based_k16_10M")
    roofline = {"bound": "hbm", "kernel": "knn_fast_kernel, stack-based k=16",
                "timed": ("cukd_knn on the queries already in Morton order, CUDA events on "
                          "the launching stream: knn_fast_kernel plus the re-run of the few "
                          "tied queries"),
                "kernel_ms": round(knn_kernel_ms, 3),
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "frac_of_whole_knn_call": round(knn_bytes / (knn_sb_ms / 1e3) / 1e9 / peak, 4),
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
        side = torch.cuda.Stream()
        e2e_q = torch.empty_like(d_q)
        # two batches in flight: one compute stream (the current one) runs
        # each step's build and search back to back; the step's points and
        # queries go up on a side stream once its slot's buffers are free;
        # each step's answers land behind its own event
        # (cukd_knn_to_host_async), so the device->host copy of one step's
        # answers (1.28 GB, the slowest stage; PCIe copies both ways at once)
        # overlaps the next step's build and search
        up_stream = torch.cuda.Stream()
        slots = []
        for j in range(2):
            slots.append({"pts": d_pts if j == 0 else torch.empty_like(d_pts),
                          "wb": wb if j == 0 else torch.empty_like(wb),
                          "ids": h_ids if j == 0 else torch.empty_like(h_ids).pin_memory(),
                          "d2": h_d2 if j == 0 else torch.empty_like(h_d2).pin_memory(),
                          "q": torch.empty((nq, 3), dtype=torch.float32, device=dev),
                          "done": torch.cuda.Event(), "free": torch.cuda.Event(),
                          "up": torch.cuda.Event(), "upq": torch.cuda.Event(), "used": False})
        step_no = [0]

        def pipelined_step():
            sl = slots[step_no[0] % 2]
            step_no[0] += 1
            main = torch.cuda.current_stream()
            if sl["used"]:
                up_stream.wait_event(sl["free"])  # the search two steps back has run
            with torch.cuda.stream(up_stream):
                sl["pts"].copy_(h_pts, non_blocking=True)
                sl["up"].record(up_stream)
                sl["q"].copy_(h_q, non_blocking=True)
                sl["upq"].record(up_stream)
            main.wait_event(sl["up"])
            ck.build_tree(sl["pts"], layout=lay, world_bounds=sl["wb"])
            if sl["used"]:
                main.wait_event(sl["done"])  # its host buffers: that step's answers landed
            main.wait_event(sl["upq"])
            sl["done"] = torch.cuda.Event(enable_timing=True)  # one per step: timed below
            ck.knn_to_host(sl["pts"], sl["q"], K, "stack_based", layout=lay,
                           world_bounds=sl["wb"], out_ids=sl["ids"], out_d2=sl["d2"],
                           chunk=args.e2e_async_chunk, done=sl["done"])
            sl["free"].record(main)
            sl["used"] = True
            return sl["done"]

        def timed_pipelined():
            for _ in range(max(2, args.warmup)):
                pipelined_step()
            barrier()
            main = torch.cuda.current_stream()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(main)
            dones = [pipelined_step() for _ in range(args.steps)]
            for sl in slots:
                main.wait_event(sl["done"])
            b.record(main)
            barrier()
            # the window opens on a drained device (the barrier synchronises),
            # so the first step's upload, build, search and answer copies run
            # back to back; the steady-state figure is the interval between
            # consecutive steps' answers landing, over the timed steps
            steady = (dones[0].elapsed_time(dones[-1]) / (args.steps - 1) if args.steps > 1
                      else a.elapsed_time(b))
            return (max_over_ranks(a.elapsed_time(b), pg, dev) / args.steps,
                    max_over_ranks(steady, pg, dev))

        def e2e_step():
            # points up, build, then cukd_knn_host: query chunks copied up,
            # searched and their answers copied down on overlapping streams
            d_pts.copy_(h_pts, non_blocking=True)
            ck.build_tree(d_pts, layout=lay, world_bounds=wb)
            ck.knn_host(d_pts, h_q, K, "stack_based", layout=lay, world_bounds=wb,
                        out_ids=h_ids, out_d2=h_d2, chunk=args.e2e_chunk)

        def device_queries_step():
            # the same inputs and outputs, the queries uploaded on a side
            # stream while the tree builds, then cukd_knn_to_host
            d_pts.copy_(h_pts, non_blocking=True)
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                e2e_q.copy_(h_q, non_blocking=True)
            ck.build_tree(d_pts, layout=lay, world_bounds=wb)
            torch.cuda.current_stream().wait_stream(side)
            ck.knn_to_host(d_pts, e2e_q, K, "stack_based", layout=lay, world_bounds=wb,
                           out_ids=h_ids, out_d2=h_d2, chunk=args.e2e_chunk)

        def timed(step):
            for _ in range(2):
                step()
            barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(args.steps):
                step()
            b.record()
            barrier()
            return max_over_ranks(a.elapsed_time(b), pg, dev) / args.steps

        et, steady_ms = timed_pipelined()
        st_ms = timed(e2e_step)
        dt = timed(device_queries_step)
        slots[1]["pts"] = slots[1]["ids"] = slots[1]["d2"] = None
        slots[0]["q"] = slots[1]["q"] = None

        # the PCIe copies alone (one whole-array copy each way, pinned host
        # memory): the floor under any e2e step that moves these bytes
        def pcie_ms(fn, reps=3):
            best = None
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                torch.cuda.synchronize()
                best = a.elapsed_time(b) if best is None else min(best, a.elapsed_time(b))
            return best
        d_res = torch.empty((nq, K), dtype=torch.int32, device=dev)
        d_tmp = torch.empty_like(d_pts)  # d_pts keeps the built tree
        up_ms = pcie_ms(lambda: (d_tmp.copy_(h_pts, non_blocking=True),
                                 e2e_q.copy_(h_q, non_blocking=True)))
        down_ms = pcie_ms(lambda: (h_ids.copy_(d_res, non_blocking=True),
                                   h_d2.view(torch.int32).copy_(d_res, non_blocking=True)))
        del d_res, d_tmp
        e2e = {"value": round(whole_job_rate(nq, world, et), 1), "unit": UNIT,
               "h2d_bytes_per_step": int(h_pts.numel() * 4 + h_q.numel() * 4),
               "d2h_bytes_per_step": int(h_ids.numel() * 4 + h_d2.numel() * 4),
               "ms_per_step": round(et, 3),
               "pcie_copies_alone_ms": {"h2d": round(up_ms, 3), "d2h": round(down_ms, 3)},
               "api": ("cukd_build_tree + cukd_knn_to_host_async (pinned host results, "
                       + (f"{args.e2e_async_chunk}-query chunks" if args.e2e_async_chunk > 0
                          else "the batch searched in one slice") +
                       ") on one stream, each step's answers copied down behind its "
                       "own event while the next step builds and searches; each step's "
                       "points and queries copied up from pinned host memory on a side "
                       "stream during the previous step; two device trees, query and answer "
                       "buffers"),
               "steady_state": {
                   "value": round(whole_job_rate(nq, world, steady_ms), 1),
                   "ms_per_step": round(steady_ms, 3),
                   "window": "the same steps: the interval between consecutive steps' answers "
                             "landing in host memory, from the first timed step's to the last's "
                             "(ms_per_step above opens on a drained device, so it also holds one "
                             "pipeline fill: the first step's upload, build, search and copies "
                             "back to back)"},
               "one_step_at_a_time": {
                   "value": round(whole_job_rate(nq, world, st_ms), 1),
                   "ms_per_step": round(st_ms, 3),
                   "api": "the same calls, every step on one stream after the previous one"},
               "device_queries_api": {
                   "value": round(whole_job_rate(nq, world, dt), 1), "ms_per_step": round(dt, 3),
                   "api": "cukd_build_tree + cukd_knn_to_host (queries uploaded on a side "
                          "stream during the build)"}}

    batched = None if args.no_batched else batched_section(ck, dev, args.batched_clouds,
                                                           args.batched_tuning)

    others = None
    if world == 1 and not args.no_configs:
        # the other configurations, each measured once (parity-test workloads
        # of the full suite): freed of this workload's buffers first
        keep_pts = d_pts.cpu().numpy() if rank == 0 and not args.no_cpu_baseline else None
        keep_wb = wb.cpu().numpy()
        del d_src, d_pts, d_q, d_ids, d_d2
        torch.cuda.empty_cache()
        others = {}
        for name, fn in (("c1", config_c1), ("c4", config_c4), ("c5", config_c5)):
            others[name] = fn(ck, dev, peak)
            torch.cuda.empty_cache()
    else:
        keep_pts = d_pts.cpu().numpy() if rank == 0 and not args.no_cpu_baseline else None
        keep_wb = wb.cpu().numpy()

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(keep_pts, keep_wb, q, step_out, learned_out)
        parity = cpu.pop("parity", None)

    out = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded Gaussian mixture, 64 components, sigma 0.01)",
           "config": bench_config(n, nq, world),
           "phases_ms": {"build": round(build_ms, 3), "knn_stack_based": round(knn_sb_ms, 3),
                         "knn_stack_free": round(knn_sf_ms, 3), "morton_order": round(morton_ms, 3),
                         "fcp_stack_based": round(fcp_ms, 3), "restore_copy": round(copy_ms, 3),
                         "knn_stack_based_reference_order": round(knn_ref_ms, 3)},
           "build_ms": round(build_ms, 3),
           "knn_stack_free_queries_per_s": round(nq / (knn_sf_ms / 1e3), 1),
           "learned_radius": learned, "batched": batched, "other_configs": others,
           "roofline": roofline, "build_roofline": build_roof,
           "cpu_baseline": cpu, "parity": parity,
           "e2e": e2e, "clocks": clocks, "gpu_launches": int(launches),
           "gpu_launches_per_step": round(launches / args.steps, 1)}
    if pg:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def batched_section(ck, dev, num_clouds=4096, tuning=""):
    """Many clouds built and queried together (cukd_batch_*): 4096 clouds of
    floor(exp(U[ln 256, ln 65536])) uniform points, 1024 uniform queries
    each, k = 8, stack-based; autotuned, then timed as CUDA-graph replays
    of build + query (the input cloud array is restored before each)."""
    import torch
    from cudakdtree_b200 import workloads as wl
    pts, poff, qs, qoff = wl.batched_clouds(num_clouds=num_clouds)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    src = torch.from_numpy(pts).to(dev)
    P = torch.empty_like(src)
    Q = torch.from_numpy(qs).to(dev)
    bnd = plan.bounds_tensor(dev)
    out = plan._outputs(dev)
    if tuning:
        t, bs, qpt, mo = (int(v) for v in tuning.split(","))
        plan.set_tuning(build_tile=t, block_size=bs, queries_per_thread=qpt, morton=mo)
        tune = plan.tuning
    else:
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
    return {"workload": f"{num_clouds} clouds, sizes floor(exp(U[ln 256, ln 65536])) (seed 5), uniform "
                        "points and 1024 uniform queries per cloud, float3, k=8, stack_based",
            "clouds": int(poff.size - 1), "points": int(n), "queries": int(nq), "k": 8,
            "tuning": {k: (round(v, 3) if isinstance(v, float) else v)
                       for k, v in tune.as_dict().items()},
            "run_ms": round(run_ms, 3), "build_ms": round(build_ms, 3),
            "query_ms": round(query_ms, 3),
            "queries_per_s": round(nq / (run_ms / 1e3), 1),
            "build_points_per_s": round(n / (build_ms / 1e3), 1),
            "kernel_launches_per_run": launches, "graph": True}


def cpu_baseline_sample(tree_records_i32, bounds, q, step_out, learned_out=None):
    """The reference's own host code (oracle/_ref) on a bounded sample of
    the workload, on this box's host cores; on the same sample, the parity
    check of this run's answers: the reference's host traversal must return
    the step's kNN ids and squared-distance bits (and the learned path's),
    and the GPU-built tree must be the reference's canonical tree (the
    oracle's canonical-tree checker, pinned to buildTree_host in the tests)."""
    try:
        from oracle import pyoracle as po
        if po.ref_host() is None:
            return {"value": None, "unit": UNIT, "unavailable": "oracle/_ref not built"}
        from cudakdtree_b200 import workloads as wl
        cores = po.nthreads()
        rec = tree_records_i32.view(po.ref_record_dtype(po.REF_F3_PACKED)).reshape(-1)
        step_ids, step_d2 = step_out
        ns = len(step_ids)
        qs = np.ascontiguousarray(q[:ns])
        t = time.perf_counter()
        ri, rd, _ = po.ref_knn_host(po.REF_F3_PACKED, rec, bounds, qs, K, po.STACK_BASED,
                                    threads=cores)
        tq = time.perf_counter() - t

        def same(out):
            return bool(np.array_equal(out[0], ri) and
                        np.array_equal(np.ascontiguousarray(out[1]).view(np.uint32),
                                       rd.view(np.uint32)))
        pay = tree_records_i32[:, 3].view(np.uint32)
        perm = (pay & 0x3FFFFFFF).astype(np.int64)
        dims = (pay >> 30).astype(np.int32)
        coords = np.ascontiguousarray(tree_records_i32[:, :3]).view(np.float32)
        is_perm = bool(np.array_equal(np.sort(perm), np.arange(len(perm))))
        violations = po.check_tree(coords, perm, dims, bounds) if is_perm else -1
        parity = {"sample_queries": ns, "knn_equal_reference": same(step_out),
                  "tree_canonical": bool(violations == 0),
                  "checker": ("reference stackBased::knn host traversal (oracle/_ref) on the "
                              "GPU-built tree; canonical-tree check of the whole tree")}
        if learned_out is not None:
            parity["learned_equal_reference"] = same(learned_out)
        parity["ok"] = all(v for key, v in parity.items()
                           if key in ("knn_equal_reference", "tree_canonical",
                                      "learned_equal_reference"))
        nb = 1_000_000
        sub = wl.packed_records(wl.gmm_points(nb, seed=3))
        sub_rec = sub.view(po.ref_record_dtype(po.REF_F3_PACKED))
        t = time.perf_counter()
        po.ref_build_host(po.REF_F3_PACKED, sub_rec)
        tb = time.perf_counter() - t
        return {"value": round(ns / tq, 1), "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": (f"reference stackBased::knn<FixedCandidateList<16>> (OpenMP, {cores} "
                           f"threads) on {ns} of the 10M queries against the full 10M-point tree "
                           "(query phase only; the tree is the GPU build, checked canonical); "
                           "reference buildTree_host on a 1M-point sample of the mixture took "
                           f"{tb:.2f} s single-threaded"),
                "build_1M_sample_s": round(tb, 3), "parity": parity}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "unavailable": repr(e)[:200],
                "parity": {"ok": False, "error": repr(e)[:200]}}


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU implementation of the path
# ---------------------------------------------------------------------------
def run_reference(args, rank, world, local):
    """The reference's own CPU code (oracle/_ref, compiled unmodified) on
    this arm's workload: cukd::buildTree_host over all points, timed once
    (single-threaded as the reference implements it, 48 s at 10M), then every
    step answers all the queries with stackBased::knn<FixedCandidateList<16>>
    in an OpenMP loop over every host thread (sampleHost.cu:58-73)."""
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
    qs = np.ascontiguousarray(q)

    def knn_step():
        t0 = time.perf_counter()
        po.ref_knn_host(po.REF_F3_PACKED, tree, bounds, qs, K, po.STACK_BASED, threads=cores)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        knn_step()
    times = [knn_step() for _ in range(args.steps)]
    step_s = float(np.mean(times))
    value = nq / step_s
    desc = (f"every step: stackBased::knn<FixedCandidateList<16>> over all {nq} queries with "
            f"{cores} OpenMP threads against the {n}-point tree; cukd::buildTree_host "
            f"(single-threaded, as the reference implements it) timed once: {t_build:.2f} s, "
            "reported as build_ms and not repeated per step")
    ref_gpu = reference_gpu_timings(recs, q)
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(step_s * 1e3, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (same seeds as our arm)",
           "config": bench_config(n, nq, world),
           "reference_step": desc,
           "build_ms": round(t_build * 1e3, 1),
           "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores,
                            "kind": "reference", "sample": desc},
           "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "reference_gpu": ref_gpu}
    print(json.dumps(out), flush=True)


def reference_gpu_timings(recs, q):
    """For context beside the CPU arm: the reference's own GPU builders and
    traversal (compiled unmodified from its headers into oracle/_ref) on the
    same records and queries, on this GPU, timed with CUDA events.  Not part
    of the arm's value."""
    try:
        import ctypes as C
        import torch
        from oracle import pyoracle as po
        if not torch.cuda.is_available() or po.ref_gpu() is None:
            return {"unavailable": "no GPU or oracle/_ref GPU library not built"}
        L = po.ref_gpu()
        n, nq = len(recs), len(q)
        src = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
        d = torch.empty_like(src)
        wb = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
        dq = torch.from_numpy(q).cuda()
        ids = torch.empty((nq, K), dtype=torch.int32, device="cuda")
        d2 = torch.empty((nq, K), dtype=torch.float32, device="cuda")

        def timed(fn):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            rc = fn()
            b.record()
            torch.cuda.synchronize()
            if rc != 0:
                raise RuntimeError(f"reference GPU call failed: {rc}")
            return a.elapsed_time(b)

        res = {}
        for builder, name in ((2, "buildTree_inPlace"), (1, "buildTree_bitonic"),
                              (0, "buildTree_thrust")):
            ts = []
            for _ in range(2):
                d.copy_(src)
                ts.append(timed(lambda: L.refg_build(po.REF_F3_PACKED, builder,
                                                     C.c_void_p(d.data_ptr()), n,
                                                     C.c_void_p(wb.data_ptr()))))
            res[name + "_ms"] = round(min(ts), 3)
            if builder == 2:  # is its output a k-d tree? (checker only)
                out = d.cpu().numpy().view(np.uint32).reshape(n, 4)
                res["buildTree_inPlace_kd_violations"] = po.check_kd(
                    out[:, :3].view(np.float32), (out[:, 3] >> 30).astype(np.int32),
                    wb.cpu().numpy())
        # the reference's spatial k-d tree builder on the same points (float3)
        pts3 = torch.from_numpy(np.ascontiguousarray(
            recs.view(np.float32).reshape(n, 4)[:, :3])).cuda()
        ms = C.c_float(0.0)
        sp = []
        for _ in range(2):
            if L.refg_spatial_build_ms_float3(C.c_void_p(pts3.data_ptr()), n, 8,
                                              C.byref(ms)) != 0:
                raise RuntimeError("reference spatial build failed")
            sp.append(ms.value)
        res["spatial_buildTree_ms"] = round(min(sp), 3)
        del pts3
        # where the reference's in-place builder's output is a valid tree:
        # 10M uniform float2 / float4 points
        from cudakdtree_b200 import workloads as wl
        for code, D in ((po.REF_F2, 2), (po.REF_F4, 4)):
            p = torch.from_numpy(wl.uniform_points(n, D, seed=7).astype(np.float32)).cuda()
            wbD = torch.zeros((2, D), dtype=torch.float32, device="cuda")
            res[f"buildTree_inPlace_uniform_float{D}_ms"] = round(timed(
                lambda: L.refg_build(code, 2, C.c_void_p(p.data_ptr()), n,
                                     C.c_void_p(wbD.data_ptr()))), 1)
            res[f"buildTree_inPlace_uniform_float{D}_kd_violations"] = po.check_kd(p.cpu().numpy())
            del p
        hb = np.ascontiguousarray(wb.cpu().numpy())
        knn = lambda: L.refg_knn(po.REF_F3_PACKED, 0, 0, K, C.c_void_p(d.data_ptr()), n,
                                 hb.ctypes.data_as(C.c_void_p), C.c_void_p(dq.data_ptr()), nq,
                                 float("inf"), C.c_void_p(ids.data_ptr()),
                                 C.c_void_p(d2.data_ptr()))
        timed(knn)
        t_knn = min(timed(knn) for _ in range(2))
        res["stackBased_knn_k16_ms"] = round(t_knn, 3)
        res["knn_queries_per_s"] = round(nq / (t_knn / 1e3), 1)
        res["build_plus_knn_queries_per_s"] = round(
            nq / ((res["buildTree_thrust_ms"] + t_knn) / 1e3), 1)
        res["note"] = ("reference code compiled unmodified with -fmad=false, one thread per "
                       "query in input order (testing/floatN-knn-and-fcp.cu pattern)")
        return res
    except Exception as e:  # context only: never fail the arm
        return {"unavailable": f"{type(e).__name__}: {e}"}


# ---------------------------------------------------------------------------
# the other configurations (parity-test workloads), measured on request
# ---------------------------------------------------------------------------
def _timer():
    import torch

    def timed(fn, reps=3, setup=None):
        if setup:
            setup()
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            if setup:
                setup()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps
    return timed


def _frac(bytes_, ms, peak):
    return round(bytes_ / (ms / 1e3) / 1e9 / peak, 4)


def _knn_bytes(ck, tree, q, k, rec_bytes, qbytes, scale=1, **kw):
    """Algorithmic bytes of a kNN launch: every node the reference's
    stack-based traversal visits read once, the queries read, (id, d2)
    written -- visits counted on `q` (a sample), scaled by `scale`."""
    v = int(ck.knn_visits(tree, q, k, "stack_based", **kw).sum().item()) * scale
    nq = q.shape[0] * scale
    return v * rec_bytes + nq * qbytes + nq * k * 8, v / nq


def config_c1(ck, dev, peak):
    """1M U[0,1)^3 float3 points (seed 1), 1M U[0,1)^3 queries (seed 2),
    round-robin dims; FCP and kNN k=8 with the three traversals; the
    reference's host build + host traversals on the same data for context."""
    import torch
    from cudakdtree_b200 import workloads as wl
    timed = _timer()
    pts = wl.uniform_points(1_000_000, seed=1)
    q = wl.uniform_points(1_000_000, seed=2)
    src = torch.from_numpy(pts).to(dev)
    P = torch.empty_like(src)
    Q = torch.from_numpy(q).to(dev)
    lay = ck.layout_for("float32", 3)
    wb = torch.empty((2, 3), dtype=torch.float32, device=dev)
    copy = lambda: P.copy_(src)
    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    build_ms = timed(lambda: ck.build_tree(P, layout=lay, world_bounds=wb), reps=5, setup=copy)
    n = len(pts)
    out = {"config": "C1", "workload": "1M uniform float3, 1M uniform queries, round-robin",
           "build_ms": round(build_ms, 3),
           "build_frac": _frac(2 * n * 12 * (int(np.log2(n)) + 1), build_ms, peak),
           "queries_per_s": {}}
    for m in ("stack_based", "stack_free", "cct"):
        t = timed(lambda: ck.fcp(P, Q, m, layout=lay, world_bounds=wb))
        out["queries_per_s"][f"fcp_{m}"] = round(len(q) / (t / 1e3), 1)
        t = timed(lambda: ck.knn(P, Q, 8, m, layout=lay, world_bounds=wb))
        out["queries_per_s"][f"knn8_{m}"] = round(len(q) / (t / 1e3), 1)
        if m == "stack_based":
            kb, mv = _knn_bytes(ck, P, Q, 8, 12, 12, layout=lay, world_bounds=wb)
            out["knn8_frac"] = _frac(kb, t, peak)
            out["knn8_mean_visits_ref"] = round(mv, 2)
    out["clocks"] = sampler.stop()
    try:
        from oracle import pyoracle as po
        if po.ref_host() is not None:
            t0 = time.perf_counter()
            tree, bounds = po.ref_build_host(po.REF_F3, pts)
            tb = time.perf_counter() - t0
            qs = np.ascontiguousarray(q[:200_000])
            t0 = time.perf_counter()
            po.ref_fcp_host(po.REF_F3, tree, bounds, qs, po.CCT)
            tf = time.perf_counter() - t0
            t0 = time.perf_counter()
            po.ref_knn_host(po.REF_F3, tree, bounds, qs, 8, po.STACK_BASED)
            tk = time.perf_counter() - t0
            out["cpu_reference"] = {"cores": po.nthreads(), "buildTree_host_ms": round(tb * 1e3, 1),
                                    "cct_fcp_queries_per_s": round(len(qs) / tf, 1),
                                    "stackBased_knn8_queries_per_s": round(len(qs) / tk, 1),
                                    "sample": "200K of the 1M queries"}
    except Exception as e:
        out["cpu_reference"] = {"unavailable": str(e)}
    return out


def config_c2(ck, dev, peak=None):
    """The benchmark workload's data with every builder name, the spatial
    tree, and kNN k=16 with the three traversals."""
    import torch
    timed = _timer()
    recs, q = workload(N_POINTS, N_QUERIES)
    n, nq = len(recs), len(q)
    lay = ck.layout_for("float32", 3, stride=RECORD_BYTES, dim_offset=12, dim_shift=30,
                        dim_bits=2)
    src = torch.from_numpy(recs.view(np.int32).reshape(n, 4).copy()).to(dev)
    P = torch.empty_like(src)
    Q = torch.from_numpy(q).to(dev)
    wb = torch.empty((2, 3), dtype=torch.float32, device=dev)
    copy = lambda: P.copy_(src)
    out = {"config": "C2", "workload": workload_desc(n, nq), "build_ms": {}, "queries_per_s": {}}
    for b in ("thrust", "bitonic", "inplace"):
        out["build_ms"][b] = round(timed(lambda: ck.build_tree(P, layout=lay, world_bounds=wb,
                                                               builder=b), setup=copy), 3)
    lay_pts = ck.layout_for("float32", 3, stride=RECORD_BYTES)
    sp = [None]

    def spatial():
        if sp[0] is not None:
            sp[0].free()
        sp[0] = ck.spatial_build(src, layout=lay_pts)
    out["build_ms"]["spatial"] = round(timed(spatial), 3)
    t = timed(lambda: sp[0].knn(Q, K, "cct"))
    out["queries_per_s"]["spatial_knn16_cct"] = round(nq / (t / 1e3), 1)
    sp[0].free()
    copy()
    ck.build_tree(P, layout=lay, world_bounds=wb)
    for m in ("stack_based", "stack_free", "cct"):
        t = timed(lambda: ck.knn(P, Q, K, m, layout=lay, world_bounds=wb))
        out["queries_per_s"][f"knn16_{m}"] = round(nq / (t / 1e3), 1)
    t = timed(lambda: ck.fcp(P, Q, "stack_based", layout=lay, world_bounds=wb))
    out["queries_per_s"]["fcp_stack_based"] = round(nq / (t / 1e3), 1)
    return out


def config_c4(ck, dev, peak):
    """Learned radius at k = 32: model trained on 1M queries of the serving
    distribution (70% mixture / 30% uniform, their own seed), then 50M such
    queries answered plain and learned."""
    import torch
    from cudakdtree_b200 import workloads as wl
    timed = _timer()
    recs, _ = workload(N_POINTS, 1)
    n = len(recs)
    lay = ck.layout_for("float32", 3, stride=RECORD_BYTES, dim_offset=12, dim_shift=30,
                        dim_bits=2)
    P = torch.from_numpy(recs.view(np.int32).reshape(n, 4).copy()).to(dev)
    wb = ck.build_tree(P, layout=lay)
    k = 32
    qtrain = torch.from_numpy(wl.mixed_queries(1_000_000, seed=14)).to(dev)
    model = ck.RadiusModel(grid_res=64, seed=1, quantile=LEARNED_QUANTILE)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    model.fit(P, qtrain, k, layout=lay, world_bounds=wb, epochs=10, batch=4096)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    nq = 50_000_000
    Q = torch.from_numpy(wl.mixed_queries(nq)).to(dev)
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d2 = torch.empty((nq, k), dtype=torch.float32, device=dev)
    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    t_plain = timed(lambda: ck.knn(P, Q, k, "stack_based", layout=lay, world_bounds=wb,
                                   out_ids=ids, out_d2=d2), reps=2)
    ref_ids = ids.clone()
    fb = [None]

    def learned():
        fb[0] = ck.knn_learned(P, Q, k, model, "stack_based", layout=lay, world_bounds=wb,
                               scale=1.2, out_ids=ids, out_d2=d2)[2]
    t_learned = timed(learned, reps=2)
    clocks = sampler.stop()
    same = bool(torch.equal(ids, ref_ids))
    kb, mv = _knn_bytes(ck, P, Q[:5_000_000], k, RECORD_BYTES, 12, scale=10, layout=lay,
                        world_bounds=wb)
    return {"config": "C4", "workload": "10M-point mixture tree, k=32, train on 1M and infer "
            "50M queries (70% mixture / 30% uniform), radius x1.2",
            "train_s": round(train_s, 3), "final_loss": round(model.final_loss, 5),
            "plain_knn_ms": round(t_plain, 3), "learned_knn_ms": round(t_learned, 3),
            "plain_queries_per_s": round(nq / (t_plain / 1e3), 1),
            "learned_queries_per_s": round(nq / (t_learned / 1e3), 1),
            "learned_speedup_vs_plain": round(t_plain / t_learned, 3),
            "plain_knn_frac": _frac(kb, t_plain, peak),
            "plain_knn_mean_visits_ref": round(mv, 2),
            "plain_knn_frac_note": "algorithmic bytes = reference stack-based visits x 16 B + "
                                   "query + answers: the uniform 30% of the queries, far from "
                                   "the mixture, make the reference order visit many nodes "
                                   "that corner culling skips, so the fraction exceeds 1",
            "fallback_rate": round(int(fb[0][0].item()) / nq, 5),
            "identical_results": same, "clocks": clocks}


# the reference's {float4 p; int dim;} record: 32 bytes (float4 is 16-byte
# aligned)
F4_STRIDE = 32


def _learned_side_by_side(ck, P, Q, k, plain_ms, ids, d2, lay, wb, n, qtrain, num_dims, grid_res):
    """The learned radius on a configuration's tree beside its plain kNN:
    trained on 1M queries of the serving distribution, radius x1.2; the
    answers must equal the plain ones (held in ids / d2)."""
    import torch
    timed = _timer()
    ref_ids, ref_d2 = ids.clone(), d2.clone()
    model = ck.RadiusModel(grid_res=grid_res, seed=1, quantile=LEARNED_QUANTILE,
                           num_dims=num_dims)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    model.fit(P, qtrain, k, layout=lay, world_bounds=wb, epochs=10, batch=4096)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    fb = [None]

    def run():
        fb[0] = ck.knn_learned(P, Q, k, model, "stack_based", layout=lay, world_bounds=wb, n=n,
                               scale=1.2, out_ids=ids, out_d2=d2)[2]
    t = timed(run, reps=1)
    same = bool(torch.equal(ids, ref_ids) and torch.equal(d2, ref_d2))
    nq = Q.shape[0]
    return {"plain_knn_ms": round(plain_ms, 3), "learned_knn_ms": round(t, 3),
            "learned_queries_per_s": round(nq / (t / 1e3), 1),
            "learned_speedup_vs_plain": round(plain_ms / t, 3),
            "fallback_rate": round(int(fb[0][0].item()) / nq, 5),
            "identical_results": same, "train_s": round(train_s, 3),
            "model": f"{num_dims}-D grid {grid_res}^{num_dims}, pinball q={LEARNED_QUANTILE}"}


def config_c5(ck, dev, peak):
    """100M float4 points (xyz U[0,1), w N(0,1)) with widest-extent dims in
    the reference's 32-byte {float4; int dim} record, and 20M int3 points in
    [-2^20, 2^20]^3 with round-robin dims; kNN k = 64 on 20M queries of each
    distribution."""
    import torch
    from cudakdtree_b200 import workloads as wl
    timed = _timer()
    out = {"config": "C5"}
    n, nq, k = 100_000_000, 20_000_000, 64
    p4 = wl.wide_float4(n, seed=7)
    rec = np.zeros((n, F4_STRIDE // 4), np.float32)
    rec[:, :4] = p4
    del p4
    lay = ck.layout_for("float32", 4, stride=F4_STRIDE, dim_offset=16)
    src = torch.from_numpy(rec.view(np.uint8).reshape(-1)).to(dev)
    del rec
    P = torch.empty_like(src)
    wb = torch.empty((2, 4), dtype=torch.float32, device=dev)
    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    bms = timed(lambda: ck.build_tree(P, layout=lay, world_bounds=wb, n=n),
                setup=lambda: P.copy_(src), reps=2)
    out["float4_100M_build_ms"] = round(bms, 3)
    out["float4_build_frac"] = _frac(2 * n * F4_STRIDE * (int(np.log2(n)) + 1), bms, peak)
    del src
    Q = torch.from_numpy(wl.wide_float4(nq, seed=9)).to(dev)
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d2 = torch.empty((nq, k), dtype=torch.float32, device=dev)
    t = timed(lambda: ck.knn(P, Q, k, "stack_based", layout=lay, world_bounds=wb, n=n,
                             out_ids=ids, out_d2=d2), reps=1)
    out["float4_knn64_queries_per_s"] = round(nq / (t / 1e3), 1)
    kb, mv = _knn_bytes(ck, P, Q[:1_000_000], k, F4_STRIDE, 16, scale=nq // 1_000_000,
                        layout=lay, world_bounds=wb, n=n)
    out["float4_knn64_frac"] = _frac(kb, t, peak)
    out["float4_learned"] = _learned_side_by_side(
        ck, P, Q, k, t, ids, d2, lay, wb, n,
        torch.from_numpy(wl.wide_float4(1_000_000, seed=11)).to(dev), num_dims=4, grid_res=32)
    del P, Q, ids, d2
    torch.cuda.empty_cache()
    pi = wl.int3_points(20_000_000, seed=8)
    qi = wl.int3_points(nq, seed=10)
    srci = torch.from_numpy(pi).to(dev)
    Pi = torch.empty_like(srci)
    layi = ck.layout_for("int32", 3)
    wbi = torch.empty((2, 3), dtype=torch.int32, device=dev)
    bms = timed(lambda: ck.build_tree(Pi, layout=layi, world_bounds=wbi),
                setup=lambda: Pi.copy_(srci), reps=2)
    out["int3_20M_build_ms"] = round(bms, 3)
    out["int3_build_frac"] = _frac(2 * len(pi) * 12 * (int(np.log2(len(pi))) + 1), bms, peak)
    Qi = torch.from_numpy(qi).to(dev)
    idsi = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d2i = torch.empty((nq, k), dtype=torch.int64, device=dev)
    t = timed(lambda: ck.knn(Pi, Qi, k, "stack_based", layout=layi, world_bounds=wbi,
                             out_ids=idsi, out_d2=d2i), reps=1)
    out["int3_knn64_queries_per_s"] = round(nq / (t / 1e3), 1)
    kb, mv = _knn_bytes(ck, Pi, Qi[:1_000_000], k, 12, 12, scale=nq // 1_000_000, layout=layi,
                        world_bounds=wbi)
    out["int3_knn64_frac"] = _frac(kb, t, peak)
    out["int3_learned"] = _learned_side_by_side(
        ck, Pi, Qi, k, t, idsi, d2i, layi, wbi, len(pi),
        torch.from_numpy(wl.int3_points(1_000_000, seed=11)).to(dev), num_dims=3, grid_res=64)
    del idsi, d2i
    out["clocks"] = sampler.stop()
    try:
        from oracle import pyoracle as po
        tree = Pi.cpu().numpy()
        qs = np.ascontiguousarray(qi[:20_000])
        t0 = time.perf_counter()
        po.knn(tree, qs, k, po.STACK_BASED, bounds=wbi.cpu().numpy())
        out["int3_cpu_restatement_knn64_queries_per_s"] = round(len(qs) / (time.perf_counter() - t0), 1)
        out["int3_cpu_note"] = (f"oracle's C restatement (the reference has no int traversal), "
                                f"{po.nthreads()} threads, 20K-query sample")
    except Exception as e:
        out["int3_cpu_restatement"] = {"unavailable": str(e)}
    return out


# ---------------------------------------------------------------------------
# small single-kernel cases (per-kernel ncu captures): inputs above the L2
# size, a few GB on the device at most; each runs its kernel(s) twice
# ---------------------------------------------------------------------------
def _gmm_tree(ck, n=10_000_000):
    import torch
    from cudakdtree_b200 import workloads as wl
    lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
    rec = torch.from_numpy(wl.packed_records(wl.gmm_points(n, seed=3)).view(np.int32)
                           .reshape(n, 4).copy()).cuda()
    return rec, ck.build_tree(rec, layout=lay), lay


def kernel_case(name):
    import torch
    import cudakdtree_b200 as ck
    from cudakdtree_b200 import workloads as wl

    def gmm_q(nq):
        return torch.from_numpy(wl.gmm_points(nq, seed=3, sample_seed=4)).cuda()
    if name == "knn":  # knn_fast_kernel: 10M-point tree, 2M queries, k = 16
        rec, wb, lay = _gmm_tree(ck)
        q = gmm_q(2_000_000)
        for _ in range(2):
            ck.knn(rec, q, 16, "stack_based", layout=lay, world_bounds=wb)
    elif name in ("learned", "train", "infer"):
        rec, wb, lay = _gmm_tree(ck)
        q = gmm_q(2_000_000)
        m = ck.RadiusModel(grid_res=64, seed=1, quantile=LEARNED_QUANTILE)
        m.fit(rec, torch.from_numpy(wl.gmm_points(1_000_000, seed=3, sample_seed=14)).cuda(),
              16, layout=lay, world_bounds=wb, epochs=2, batch=4096)
        for _ in range(2):
            if name == "infer":
                m.predict(q)
            else:
                ck.knn_learned(rec, q, 16, m, "stack_based", layout=lay, world_bounds=wb,
                               scale=1.2)
    elif name == "heap":  # k = 64: knn_fast_heap_kernel
        rec, wb, lay = _gmm_tree(ck)
        q = gmm_q(1_000_000)
        for _ in range(2):
            ck.knn(rec, q, 64, "stack_based", layout=lay, world_bounds=wb)
    elif name == "fastint":  # 20M int3 points, k = 64
        p = torch.from_numpy(wl.int3_points(20_000_000)).cuda()
        wb = ck.build_tree(p)
        q = torch.from_numpy(wl.int3_points(1_000_000, seed=9)).cuda()
        for _ in range(2):
            ck.knn(p, q, 64, world_bounds=wb)
    elif name == "accumulate":  # sharded kNN fold: two 2M-point shards
        from cudakdtree_b200 import shard
        pts = wl.gmm_points(4_000_000, seed=3)
        for _ in range(2):
            shard.sharded_knn([torch.from_numpy(pts[:2_000_000]).cuda(),
                               torch.from_numpy(pts[2_000_000:]).cuda()], 16)
    elif name == "spatial":  # spatial tree over 10M points, kNN k = 16 (cct)
        pts = torch.from_numpy(wl.gmm_points(10_000_000, seed=3)).cuda()
        q = gmm_q(2_000_000)
        t = None
        for _ in range(2):
            if t is not None:
                t.free()
            t = ck.spatial_build(pts)
            t.knn(q, 16, "cct")
    elif name == "scatter":  # Morton order of 10M queries
        q = torch.from_numpy(wl.gmm_points(10_000_000, seed=3, sample_seed=4)).cuda()
        for _ in range(2):
            ck.morton_order(q)
    elif name in ("build", "inplace", "bitonic"):  # the benchmark's 10M-point build
        lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
        src = torch.from_numpy(wl.packed_records(wl.gmm_points(10_000_000, seed=3))
                               .view(np.int32).reshape(-1, 4).copy()).cuda()
        d = torch.empty_like(src)
        for _ in range(2):
            d.copy_(src)
            ck.build_tree(d, layout=lay, builder="default" if name == "build" else name)
        ck.build_check()
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": name, "ok": True}))


KERNEL_CASES = ("knn", "learned", "train", "infer", "heap", "fastint", "accumulate", "spatial",
                "scatter", "build", "inplace", "bitonic")


def config_builders(ck, dev, peak=None):
    """Every builder name on 10M uniform float2 / float3 / float4 points and
    on the benchmark's 10M mixture records: build ms (fresh copy of the
    input before each build, mean of three)."""
    import torch
    from cudakdtree_b200 import workloads as wl
    timed = _timer()
    out = {"config": "builders", "build_ms": {}}
    cases = [(f"uniform10M_float{D}", torch.from_numpy(wl.uniform_points(10_000_000, D, seed=7)
                                                      .astype(np.float32)).to(dev), None)
             for D in (2, 3, 4)]
    recs, _ = workload(N_POINTS, 1)
    cases.append(("gmm10M_packed16", torch.from_numpy(recs.view(np.int32).reshape(-1, 4).copy())
                  .to(dev), ck.layout_for("float32", 3, stride=RECORD_BYTES, dim_offset=12,
                                          dim_shift=30, dim_bits=2)))
    for name, src, lay in cases:
        P = torch.empty_like(src)
        copy = lambda: P.copy_(src)
        for b in ("default", "bitonic", "inplace"):
            out["build_ms"][f"{name}_{b}"] = round(timed(
                lambda: ck.build_tree(P, layout=lay, builder=b), setup=copy), 3)
        ck.build_check()
    return out


def run_configs(args):
    import torch
    import cudakdtree_b200 as ck
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    fns = {"c1": config_c1, "c2": config_c2, "c4": config_c4, "c5": config_c5,
           "builders": config_builders}
    peak, _ = measured_peaks()
    for name in [c.strip().lower() for c in args.configs.split(",") if c.strip()]:
        res = fns[name](ck, dev, peak)
        print(json.dumps(res), flush=True)
        torch.cuda.empty_cache()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.kernel_case:
        kernel_case(args.kernel_case)
        return
    if args.configs:
        if rank == 0:
            run_configs(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
