#!/usr/bin/env python
"""Benchmark of the TagMatch subset-matching hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (config1 shapes): 10,000,000 stored 192-bit filters from the seeded
generator (seed 2, tag sets of 1-8 Zipf(1.0) tags over 100,000 tags, 7 bits
per tag, 1-4 keys per filter), partitions of at most 65,536 filters, and
1,000,000 queries per GPU per step, matched in per-partition batches of 256
queries.  A step is one pass of `match` over the step's queries.

* value: queries/s with the queries already resident in HBM (device API),
  timed with CUDA events on the matcher's stream, max over ranks.
* e2e: the same through the host C ABI (tm_match_batch): host->device copy
  of the queries and device->host copy of every result key inside the timed
  region.
* roofline: the subset-test kernel's algorithmic bytes per launch over its
  CUDA-event duration, against the measured HBM copy bandwidth.
* cpu_baseline: the oracle's C port of the reference matcher on this host's
  cores, on a bounded sample of the same queries.

--impl reference times the reference's own sequential matcher (test_matcher,
built from the reference sources into oracle/_ref), one process per host
core over shards of a query sample, on the same table.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "queries/s at 10M 192-bit filters (bit-exact) and p50/p99 latency vs plain GPU"
UNIT = "queries/s"
FILTERS = 10_000_000
QUERIES = 1_000_000
SEED = 2
MAX_P = 65_536
L2_BYTES = 126 * 1024 * 1024
# queries that share one pass of the subset test over a partition's tiles
# (a work item: four 256-query chunks)
ITEM_QUERIES = 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1, choices=[1, 2],
                    help="1: 10M filters (the headline); 2: 100M filters, Zipf s=1.3, superset fractions 10/50/90%%")
    ap.add_argument("--filters", type=int, default=FILTERS)
    ap.add_argument("--queries", type=int, default=QUERIES)
    ap.add_argument("--batch", type=int, default=131072, help="queries per device batch")
    ap.add_argument("--unique", action="store_true", help="time match_unique instead of match")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--seg-tiles", type=int, default=0, help="tiles per work item (instead of autotuning)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--parity-samples", type=int, default=2000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-rates", default="250000,500000,750000,1000000,1500000")
    ap.add_argument("--serve-plain-rates", default="100000,200000,300000,450000,600000")
    ap.add_argument("--serve-modes", default="plain,continuous,learned")
    ap.add_argument("--serve-results", default="host,device")
    ap.add_argument("--latency-target-ms", type=int, default=25)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned work-queue order comparison")
    ap.add_argument("--no-small-partitions", action="store_true",
                    help="config 2: skip the small-partition CPU backend comparison")
    ap.add_argument("--small-threshold", type=int, default=1024, help="config 2: partitions below this many filters")
    ap.add_argument("--small-queries", type=int, default=32768, help="config 2: queries of that comparison")
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            rows = open(self.path).read().strip().splitlines()
        except OSError:
            rows = []
        for r in rows:
            t = [x.strip() for x in r.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx.append(float(t[2]))
            except ValueError:
                continue
            for n, v in zip(names, t[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if self.path:
            os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kw = {}
        if backend == "nccl":
            import torch
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900), **kw)
    return world, rank, local


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def shard_seed(rank):
    """Rank 0 matches the configuration's own query stream; others get their own."""
    return SEED if rank == 0 else SEED + 7919 * rank


def cpu_baseline(f, ko, k, q, seconds, unique=False):
    """The oracle's C port of test_matcher on all host cores, bounded sample:
    one scan of the table per query with its keys gathered (the work of
    test_matcher.cc:74-81), reduced to a digest instead of printed."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    n = max(cores, 8)
    t0 = time.perf_counter()
    oracle.match_digest(f, ko, k, q[:n], unique=unique, threads=cores)
    dt = time.perf_counter() - t0
    per_q = dt / n
    m = int(min(q.shape[0], max(n, seconds / max(per_q, 1e-9))))
    t0 = time.perf_counter()
    oracle.match_digest(f, ko, k, q[:m], unique=unique, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": m / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {m} of the step's queries against the full {f.shape[0]}-filter table, one pass per "
                      f"query (oracle/oracle.c restatement of test_matcher.cc:74-81), {dt:.1f} s"}


def parity_check(tm, f, ko, k, q, base, B, unique, stream, samples):
    """Checks the timed configuration itself: one more step with the same
    tiles per work item and device batch; every (nq / samples)-th query's
    keys are read back from the device and digested (count, multiset hash),
    against the oracle's single-pass matcher on the same table."""
    from oracle import oracle
    from tagmatch_b200.tagmatch import read_device
    nq = q.shape[0]
    stride = max(1, nq // samples)
    sel = np.arange(0, nq, stride)
    got_c = np.zeros(sel.size, dtype=np.uint64)
    got_h = np.zeros(sel.size, dtype=np.uint64)
    j = 0
    for b0 in range(0, nq, B):
        n = min(B, nq - b0)
        po, pk, _ = tm.match_batch_device(base + b0 * 24, n, unique=unique, stream=stream)
        off = read_device(po, n + 1, np.uint64)
        while j < sel.size and sel[j] < b0 + n:
            i = int(sel[j]) - b0
            keys = read_device(pk + int(off[i]) * 4, int(off[i + 1] - off[i]), np.uint32)
            c, h = oracle.digest(np.array([0, keys.size], dtype=np.uint64), keys)
            got_c[j], got_h[j] = c[0], h[0]
            j += 1
    t0 = time.perf_counter()
    exp_c, exp_h = oracle.match_digest(f, ko, k, q[sel], unique=unique)
    bad = int(np.count_nonzero((exp_c != got_c) | (exp_h != got_h)))
    return {"checked": int(sel.size), "mismatches": bad, "every": int(stride),
            "keys_checked": int(got_c.sum()), "oracle_s": round(time.perf_counter() - t0, 1),
            "how": "per-query (count, multiset hash) of the device results of one more step at the timed "
                   "configuration, against oracle/oracle.c's single-pass restatement of test_matcher.cc:74-81"
                   + (" + tagmatch_query.hh:99-119 sort/unique" if unique else "")}


def learned_order(tm, step, args, stream):
    """The learned scheduler on the timed workload: two steps recorded as
    timing samples, the cost model trained on the GPU, then steps with the
    work queue in the model's order against steps in partition id order
    (alternating, CUDA events on the matcher's stream)."""
    import torch
    tm.sched_record(True)
    for _ in range(2):
        step()
    tm.sched_record(False)
    rep = tm.sched_train(epochs=30)
    times = {False: [], True: []}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(2 * max(2, args.steps)):
        use = bool(i & 1)
        tm.sched_use_order(use)
        torch.cuda.synchronize()
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        times[use].append(e0.elapsed_time(e1))
    tm.sched_use_order(False)
    static_ms, learned_ms = statistics.median(times[False]), statistics.median(times[True])
    return {"model": "8-64-64-1 fp32 MLP, trained by the library's kernels on per-item timing samples",
            "samples": rep["samples"], "train_steps": rep["steps"], "train_ms": round(rep["ms"], 1),
            "val_r2": round(rep["val_r2"], 4), "val_mse": round(rep["val_mse"], 4), "mean_mse": round(rep["mean_mse"], 4),
            "static_order_ms_per_step": round(static_ms, 3), "learned_order_ms_per_step": round(learned_ms, 3),
            "gain": round(static_ms / learned_ms - 1.0, 4),
            "pred_batch_ms": {str(b): round(tm.sched_predict_batch_ms(b), 3) for b in (1024, 16384, 131072)}}


def serving(args):
    """Latency under a Poisson load of 1..4096-query requests (C++ driver over
    tm_submit): plain = one request per device batch, continuous = pending
    requests share batches on two lanes, learned = continuous batching with
    the learned scheduler's flush points (trained on a calibration load)."""
    from tagmatch_b200 import build
    cmd = [build.SERVE_BENCH, f"filters={args.filters}", "pool=1048576", f"seed={SEED}", f"maxp={MAX_P}",
           f"rates={args.serve_rates}", f"plain_rates={args.serve_plain_rates}", f"modes={args.serve_modes}",
           f"seconds={args.serve_seconds}", f"target_ms={args.latency_target_ms}", f"results={args.serve_results}"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        return {"error": out.stderr[-500:]}
    runs = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    return {"workload": "Poisson arrivals, request sizes log-uniform 1..4096 queries, 10M-filter table, match; "
                        "results copied to host memory (host) or left in device memory (device)",
            "runs": runs,
            "equal_p99": {res: equal_p99([r for r in runs if r.get("results") == res])
                          for res in args.serve_results.split(",")}}


def equal_p99(runs, levels=(10, 15, 20, 25, 30, 40, 50)):
    """Sustained queries/s of each mode at equal p99 latency: for each p99
    level, the highest sustained rate among the mode's runs whose p99 is at
    or below it (no interpolation), and the ratios to the plain mode."""
    modes = sorted({r["mode"] for r in runs if "p99_ms" in r})
    out = []
    for lv in levels:
        best = {m: max([r["sustained_qps"] for r in runs if r.get("mode") == m and r["p99_ms"] <= lv], default=None)
                for m in modes}
        row = {"p99_ms_at_most": lv, **{m: best[m] for m in modes}}
        if best.get("plain"):
            for m in modes:
                if m != "plain" and best[m]:
                    row[f"{m}_over_plain"] = round(best[m] / best["plain"], 2)
        out.append(row)
    return out


def run_config2(args):
    """The skewed configuration: 100,000,000 filters with Zipf s = 1.3 tags
    (seed 3; partition sizes from 1 to 65,536, heavily uneven), queries at
    superset fractions 10%, 50% and 90% (--queries per fraction).  A step is
    one pass over all three fractions' queries; per fraction: queries/s,
    keys per query, work items per batch, and the item tail (largest and
    99th-percentile item warp-cycles over the mean, from one recorded
    batch).  Tiles per work item and the device batch are autotuned on the
    50% fraction, the batch capped so that its results fit in memory."""
    import torch
    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    from tagmatch_b200 import TagMatch, workload
    n_f = args.filters if args.filters != FILTERS else 100_000_000
    t0 = time.perf_counter()
    f, ko, k = workload.generate_filters(n_f, 3, zipf_s=1.3)
    fractions = (0.1, 0.5, 0.9)
    qs = {s: workload.generate_queries(args.queries, f, 3 + 7919 * rank, zipf_s=1.3, superset_fraction=s)
          for s in fractions}
    t_gen = time.perf_counter() - t0
    tm = TagMatch()
    tm.set_persistence(False)
    t0 = time.perf_counter()
    tm.add_many(f, ko, k)
    tm.consolidate(MAX_P, 1)
    t_build = time.perf_counter() - t0
    info = tm.table_info()
    stream = torch.cuda.current_stream()
    dqs = {s: torch.from_numpy(qs[s].view(np.int32)).to("cuda") for s in fractions}
    nq = args.queries
    # keys per query on a small sample bound the device batch
    _, _, nk = tm.match_batch_device(dqs[0.9].data_ptr(), min(nq, 2048), stream=stream.cuda_stream)
    kpq = max(1.0, nk / min(nq, 2048))
    cap = int(min(262144, max(1024, 24e9 / (kpq * 9.0))))
    cap = 1 << (cap.bit_length() - 1)
    tm.set_batch_limit(cap)
    tuned = None
    B = min(args.batch, cap)
    if args.seg_tiles:
        tm.set_tiles_per_item(args.seg_tiles)
    elif not args.no_autotune:
        seg, bl, tqps = tm.autotune(qs[0.5][: min(nq, cap)])
        B = min(bl, cap)
        tuned = {"seg_tiles": seg, "device_batch": bl, "sample_queries_per_s": round(tqps, 1)}

    def step_one(s):
        keys = 0
        for b0 in range(0, nq, B):
            _, _, n = tm.match_batch_device(dqs[s].data_ptr() + b0 * 24, min(B, nq - b0), stream=stream.cuda_stream)
            keys += n
        return keys

    for s in fractions:  # warm-up: one device batch per fraction, three times
        for _ in range(max(3, args.warmup)):
            tm.match_batch_device(dqs[s].data_ptr(), min(B, nq), stream=stream.cuda_stream)
    tm.reset_match_stats()
    tm.set_profiling(True)
    per = {s: {"ms": 0.0, "keys": 0} for s in fractions}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            for s in fractions:
                e0.record(stream)
                per[s]["keys"] += step_one(s)
                e1.record(stream)
                torch.cuda.synchronize()
                per[s]["ms"] += e0.elapsed_time(e1)
    tm.set_profiling(False)
    total_ms = sum(per[s]["ms"] for s in fractions) / args.steps
    ms_max = max_over_ranks(total_ms, world, device="cuda")
    st = tm.match_stats()
    rows = []
    for s in fractions:
        tm.sched_record(True)
        tm.match_batch_device(dqs[s].data_ptr(), min(B, nq), stream=stream.cuda_stream)
        tm.sched_record(False)
        _, lc = tm.sched_samples()
        cyc = np.exp(lc[-max(1, min(lc.size, 1 << 20)):].astype(np.float64)) if lc.size else np.ones(1)
        rows.append({"superset_fraction": s, "queries_per_s": round(args.steps * nq / (per[s]["ms"] / 1e3), 1),
                     "ms_per_pass": round(per[s]["ms"] / args.steps, 2),
                     "keys_per_query": round(per[s]["keys"] / (args.steps * nq), 1),
                     "items_in_recorded_batch": int(cyc.size),
                     "item_tail": {"max_over_mean": round(float(cyc.max() / cyc.mean()), 2),
                                   "p99_over_mean": round(float(np.percentile(cyc, 99) / cyc.mean()), 2)}})
    launches = max(st["match_kernel_launches"], 1)
    alg_bytes = (st["dense_tests"] * 24 / ITEM_QUERIES + st["routed"] * 24 + st["records"] * 16) / launches
    kern_s = st["match_kernel_ms"] / 1e3 / launches
    peak, peak_kind = measured_peaks()
    line = {"metric": METRIC, "value": round(world * 3 * nq / (ms_max / 1e3), 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms_max, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"config2: {n_f} filters, Zipf s=1.3 tags (seed 3), {nq} queries per superset "
                                   f"fraction 10/50/90%, partitions <= {MAX_P}, 256-query partition batches, match",
                       "filters": n_f, "queries_per_fraction": nq, "device_batch": B, "batch_cap": cap,
                       "autotuned": tuned, "seg_tiles": tm.get_tiles_per_item(), "partitions": info["partitions"],
                       "tiles": info["tiles"], "table_device_bytes": info["device_bytes"],
                       "parallelism": f"replicas x{world}", "build_s": round(t_build, 1), "gen_s": round(t_gen, 1)},
            "clocks": clk.summary(), "gpu_launches": int(st["kernel_launches"]), "fractions": rows,
            "roofline": {"bound": "hbm", "achieved": round(alg_bytes / kern_s / 1e9, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(alg_bytes / kern_s / 1e9 / peak, 4), "traffic": None, "peak_source": peak_kind,
                         "kernel": "k_match (subset test)", "kernel_ms_per_launch": round(kern_s * 1e3, 3),
                         "alg_bytes_per_launch": int(alg_bytes)}}
    if rank == 0 and not args.no_parity:
        par = []
        for s in fractions:
            p = parity_check(tm, f, ko, k, qs[s][: min(nq, B)], dqs[s].data_ptr(), B, False, stream.cuda_stream,
                             max(16, args.parity_samples // 10))
            par.append({"superset_fraction": s, "checked": p["checked"], "mismatches": p["mismatches"]})
        line["parity"] = {"checked": sum(p["checked"] for p in par), "mismatches": sum(p["mismatches"] for p in par),
                          "per_fraction": par, "seg_tiles": tm.get_tiles_per_item(), "device_batch": B}
    if rank == 0 and world == 1 and not args.no_small_partitions:
        line["small_partitions"] = small_partition_comparison(f, ko, k, qs[0.5], dqs[0.5], args, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    tm.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def small_partition_comparison(f, ko, k, q, dq, args, stream):
    """The reference's small-partition CPU backend (back_end.cc:496-517) as a
    measured comparison, not a fallback: the partitions of the table below
    --small-threshold filters, one batch of queries routed to them by mask;
    the CPU restatement of that backend on all host cores against the GPU
    engine on a table of the same filters; parity of per-query digests."""
    import torch

    from oracle import oracle
    from tagmatch_b200 import TagMatch, balanced_partitioning
    from tagmatch_b200.tagmatch import read_device
    nq = min(q.shape[0], args.small_queries)
    q = q[:nq]
    part_of, masks, sizes = balanced_partitioning(f, MAX_P)
    small = np.nonzero(sizes < args.small_threshold)[0]
    if small.size == 0:
        return {"partitions": 0}
    is_small = np.zeros(sizes.size, dtype=bool)
    is_small[small] = True
    sel = np.nonzero(is_small[part_of])[0]
    sel = sel[np.argsort(part_of[sel], kind="stable")]
    remap = np.full(sizes.size, -1, dtype=np.int64)
    remap[small] = np.arange(small.size)
    part_off = np.zeros(small.size + 1, dtype=np.uint32)
    np.add.at(part_off, remap[part_of[sel]] + 1, 1)
    part_off = np.cumsum(part_off).astype(np.uint32)
    fg = np.ascontiguousarray(f[sel])
    lens = (ko[1:] - ko[:-1])[sel].astype(np.int64)
    kg_off = np.zeros(sel.size + 1, dtype=np.uint32)
    kg_off[1:] = np.cumsum(lens)
    starts = ko[sel].astype(np.int64)
    pos = np.repeat(starts - kg_off[:-1].astype(np.int64), lens) + np.arange(int(kg_off[-1]), dtype=np.int64)
    kg = k[pos]
    route_off, routed = oracle.route(masks[small], q)
    pair_tests = int(np.sum((part_off[1:] - part_off[:-1]).astype(np.int64) * (route_off[1:] - route_off[:-1])))
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    cc, ch = oracle.cpu_backend(fg, part_off, kg_off, kg, q, route_off, routed, threads=cores)
    cpu_s = time.perf_counter() - t0
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(fg, kg_off, kg)
    tm.consolidate(MAX_P, 1)
    tm.match_batch_device(dq.data_ptr(), nq, stream=stream.cuda_stream)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(3):
        e0.record(stream)
        po, pk, _ = tm.match_batch_device(dq.data_ptr(), nq, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    off = read_device(po, nq + 1, np.uint64)
    samp = np.arange(0, nq, max(1, nq // 512))
    bad = 0
    for i in samp:
        keys = read_device(pk + int(off[i]) * 4, int(off[i + 1] - off[i]), np.uint32)
        c, h = oracle.digest(np.array([0, keys.size], dtype=np.uint64), keys)
        bad += int(c[0] != cc[i] or h[0] != ch[i])
    tm.close()
    gpu_s = statistics.median(ms) / 1e3
    return {"threshold_filters": args.small_threshold, "partitions": int(small.size), "filters": int(sel.size),
            "queries": nq, "routed_pairs": int(routed.size), "filter_query_tests": pair_tests,
            "cpu_backend": {"s": round(cpu_s, 3), "queries_per_s": round(nq / cpu_s, 1), "cores": cores,
                            "tests_per_s": round(pair_tests / cpu_s, 1),
                            "how": "oracle/oracle.c restatement of back_end.cc:496-517 (every filter of the "
                                   "partition against every routed query), partitions over all host threads"},
            "gpu": {"s": round(gpu_s, 5), "queries_per_s": round(nq / gpu_s, 1),
                    "how": "tm_match_batch_device on a table of the same filters (re-partitioned by the engine)"},
            "gpu_over_cpu": round(cpu_s / gpu_s, 1),
            "parity": {"checked": int(samp.size), "mismatches": bad}}


def run_ours(args):
    import torch
    world, rank, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    from tagmatch_b200 import TagMatch, workload

    t0 = time.perf_counter()
    f, ko, k = workload.generate_filters(args.filters, SEED)
    q = workload.generate_queries(args.queries, f, shard_seed(rank))
    t_gen = time.perf_counter() - t0
    tm = TagMatch()
    tm.set_persistence(False)
    t0 = time.perf_counter()
    tm.add_many(f, ko, k)
    tm.consolidate(MAX_P, 1)
    t_build = time.perf_counter() - t0
    info = tm.table_info()

    stream = torch.cuda.current_stream()
    dq = torch.from_numpy(q.view(np.int32)).to("cuda")
    base = dq.data_ptr()
    nq = q.shape[0]
    B = args.batch
    tuned = None
    if args.seg_tiles:
        tm.set_tiles_per_item(args.seg_tiles)
    elif not args.no_autotune:
        # tiles per work item and device batch size, timed on a sample
        seg, bl, tqps = tm.autotune(q[: min(nq, 262144)])
        B = bl
        tuned = {"seg_tiles": seg, "device_batch": bl, "sample_queries_per_s": round(tqps, 1)}

    def step():
        keys = 0
        for b0 in range(0, nq, B):
            n = min(B, nq - b0)
            _, _, nk = tm.match_batch_device(base + b0 * 24, n, unique=args.unique, stream=stream.cuda_stream)
            keys += nk
        return keys

    for _ in range(args.warmup):
        step_keys = step()
    tm.reset_match_stats()
    tm.set_profiling(True)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step_keys = step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    tm.set_profiling(False)
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = max_over_ranks(ms, world, device="cuda")
    st = tm.match_stats()
    clocks = clk.summary()

    # roofline of the subset-test kernel: algorithmic bytes per launch over
    # its event-timed duration: the partition's filters (24 B each) once per
    # work item of ITEM_QUERIES queries, 24 B per routed query, 16 B per hit
    # record written
    launches = max(st["match_kernel_launches"], 1)
    alg_bytes = (st["dense_tests"] * 24 / ITEM_QUERIES + st["routed"] * 24 + st["records"] * 16) / launches
    kern_s = st["match_kernel_ms"] / 1e3 / launches
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / kern_s / 1e9
    traffic = None
    issue = None
    prof = os.path.join(ROOT, "profiles", "k_match_traffic.txt")
    if os.path.exists(prof):
        kv = dict(l.strip().split("=", 1) for l in open(prof) if "=" in l and not l.startswith("#"))
        # the captured case is smaller than a full launch; scale by queries
        traffic = round(float(kv["dram_bytes"]) * (st["queries"] / launches) / float(kv["queries_per_launch"]))
        if "alu_pipe_frac" in kv:
            issue = {"alu_pipe_frac": float(kv["alu_pipe_frac"]), "issue_active_frac": float(kv["issue_active_frac"]),
                     "source": "ncu --set full of one 16,384-query launch (profiles/k_match_config1_small.md)"}
    int_ops = 6 * st["dense_tests"] / launches
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_source": peak_kind,
                "kernel": "k_match (subset test)", "kernel_ms_per_launch": round(kern_s * 1e3, 3),
                "alg_bytes_per_launch": int(alg_bytes),
                "dense_word_tests_per_s": round(int_ops / kern_s / 1e12, 2),
                "dense_word_tests_unit": "T/s (6 per routed (query, filter) pair, before tile pruning)",
                "binding": "instruction issue (integer ALU pipe); DRAM is not the limit", "issue": issue}

    line = {"metric": METRIC, "value": round(world * nq / (ms_max / 1e3), 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator)",
            "config": {"workload": f"config1: {args.filters} filters (seed 2), {nq} queries/step/GPU, "
                                   f"partitions <= {MAX_P}, 256-query partition batches, "
                                   f"{'match_unique' if args.unique else 'match'}",
                       "filters": args.filters, "queries_per_step_per_gpu": nq, "device_batch": B,
                       "autotuned": tuned,
                       "partitions": info["partitions"], "tiles": info["tiles"],
                       "table_device_bytes": info["device_bytes"],
                       "l2": "inputs larger than L2 (table %.0f MB + per-step queues and results)" % (
                           info["device_bytes"] / 2**20),
                       "parallelism": f"replicas x{world}", "build_s": round(t_build, 2), "gen_s": round(t_gen, 2)},
            "clocks": clocks, "gpu_launches": int(st["kernel_launches"]), "roofline": roofline,
            "matches": {"routed_per_query": round(st["routed"] / max(st["queries"], 1), 2),
                        "pairs_per_query": round(st["pairs"] / max(st["queries"], 1), 2),
                        "hit_records_per_query": round(st["records"] / max(st["queries"], 1), 2),
                        "keys_per_query": round(st["keys"] / max(st["queries"], 1), 2)}}

    line["config"]["seg_tiles"] = tm.get_tiles_per_item()
    if rank == 0 and not args.no_parity:
        line["parity"] = parity_check(tm, f, ko, k, q, base, B, args.unique, stream.cuda_stream, args.parity_samples)
        line["parity"].update({"seg_tiles": tm.get_tiles_per_item(), "device_batch": B})
    if rank == 0 and world == 1 and not args.no_learned:
        line["learned_scheduler"] = learned_order(tm, step, args, stream)

    # ---- end to end through the host C ABI ----
    if not args.no_e2e:
        tm.set_batch_limit(B)
        qh = torch.from_numpy(q.view(np.int32)).pin_memory().numpy().view(np.uint32)
        need = int(step_keys * 1.05) + 1024
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = None
        e2e_nq = nq
        # the ranks of this node share its memory
        local_ranks = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        budget = 0.6 * avail / max(local_ranks, 1) if avail is not None else None
        if budget is not None and need * 4 > budget:
            e2e_nq = max(min(B, nq), int(nq * budget / (need * 4)))
            need = int(need * e2e_nq / nq) + 1024
        # caller-owned pinned output (the result keys of a whole step)
        out_keys = torch.empty(need, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        out_off = torch.empty(e2e_nq + 1, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        import ctypes

        from tagmatch_b200 import _native
        lib = _native.load()
        nk = ctypes.c_uint64(0)

        def e2e_step():
            s = lib.tm_match_batch(tm._h, qh[:e2e_nq].ctypes.data_as(_native.u32p), e2e_nq, 1 if args.unique else 0,
                                   out_off.ctypes.data_as(_native.u64p), out_keys.ctypes.data_as(_native.u32p),
                                   out_keys.size, ctypes.byref(nk))
            if s != 0:
                raise RuntimeError(f"tm_match_batch failed: {s}")

        e2e_step()
        barrier(world)
        tm.reset_match_stats()
        t0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            e2e_step()
        dt = (time.perf_counter() - t0) / e2e_steps
        dt = max_over_ranks(dt, world, device="cuda")
        est = tm.match_stats()
        line["e2e"] = {"value": round(world * e2e_nq / dt, 1), "unit": UNIT,
                       "h2d_bytes_per_step": int(est["h2d_bytes"] // e2e_steps),
                       "d2h_bytes_per_step": int(est["d2h_bytes"] // e2e_steps), "queries_per_step": e2e_nq,
                       "keys_per_step": int(nk.value),
                       "api": "tm_match_batch (pinned host input and output buffers)"}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(f, ko, k, q, args.cpu_seconds, args.unique)
    if rank == 0 and world == 1 and not args.no_serve:
        line["serving"] = serving(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    tm.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    world, rank, local = dist_setup("gloo")
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    from oracle import oracle
    from tagmatch_b200 import workload
    if not os.path.exists(oracle.REF_MATCHER):
        print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT,
                          "unavailable": "oracle/_ref/test_matcher was not built from the reference sources"}))
        return
    f, ko, k = workload.generate_filters(args.filters, SEED)
    q = workload.generate_queries(max(args.queries, 1), f, SEED)
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        fp = os.path.join(d, "filters.bin")
        oracle.write_partition_fib(fp, f, ko, k)
        empty = os.path.join(d, "empty.bin")
        open(empty, "wb").close()

        def run_shards(per_proc, offset):
            files = []
            for c in range(cores):
                qp = os.path.join(d, f"q{c}.bin")
                lo = offset + c * per_proc
                np.ascontiguousarray(q[lo % q.shape[0]:][:per_proc], dtype="<u4").tofile(qp)
                files.append(qp)
            t0 = time.perf_counter()
            procs = [subprocess.Popen([oracle.REF_MATCHER, "F=" + fp, "Q=" + qp], stdout=subprocess.DEVNULL)
                     for qp in files]
            for p in procs:
                p.wait()
            return time.perf_counter() - t0

        # table load time of test_matcher (no queries), subtracted from every
        # step; measured twice, the first run warming the file cache
        for _ in range(2):
            t0 = time.perf_counter()
            procs = [subprocess.Popen([oracle.REF_MATCHER, "F=" + fp, "Q=" + empty], stdout=subprocess.DEVNULL)
                     for _ in range(cores)]
            for p in procs:
                p.wait()
            t_load = time.perf_counter() - t0
        # calibrate queries per process for ~10 s of matching per step: a
        # probe long enough (24 queries, ~1.6 s at 10M filters) to stand
        # above the noise of the subtracted table load
        probe = 24
        t = max(run_shards(probe, 0) - t_load, 0.3)
        per = int(max(8, min(512, probe * 10.0 / t)))
        for w in range(args.warmup):
            run_shards(per, (w + 1) * per * cores)
        times = []
        for s in range(args.steps):
            times.append(max(1e-6, run_shards(per, (args.warmup + s + 1) * per * cores) - t_load))
    v = per * cores / statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * statistics.mean(times), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"config1: {args.filters} filters (seed 2), {per * cores} sampled queries/step",
                       "filters": args.filters},
            "cpu_baseline": {"value": round(v, 2), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{per} queries x {cores} test_matcher processes per step; "
                                       f"table load ({t_load:.1f} s) subtracted"},
            "e2e": {"value": round(v, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == 2:
        run_config2(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
