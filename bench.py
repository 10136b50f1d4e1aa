#!/usr/bin/env python
"""Benchmark: continuous subgraph matching on one B200.

Default workload (--config 4, the serving loop at full size; seeded and
synthetic, the reference's dataset is not available): R-MAT(0.57, 0.19,
0.19) with 2^24 vertices and 2^28 undirected edges (10 % withheld for
re-insertion), 32 uniform vertex labels; update requests of lognormal size
(median 512, capped at 65,536 updates), 60 % inserts / 40 % deletes; a pool
of 64 random-walk queries of 4-10 vertices, all registered at the start, and
query churn: every 4th request arrives with a registration (a pool query) or
a retirement (an initial query), alternately.

The same requests, arrival times and churn run through three forms of the
engine, each from the same initial graph (between forms the graph is put
back by applying the inverse of every effective update, without matching):
  served:  the serving loop -- continuous batching of queued requests into one
           device batch, host assembly of batch k overlapping device batch
           k + 1, each device batch replayed from captured CUDA graphs;
  batched: one request at a time, every registered query in one persistent
           matcher launch (DSM_OPT_PLAIN = 0), no overlap;
  plain:   one request at a time, one matcher launch per query with a host
           round trip after each -- the reference's one-query-per-process loop.
Every form lists the per-update positive / negative embeddings (canonically
sorted).  Each (query, update) search is bounded by DSM_OPT_WORK_LIMIT
(partial embeddings generated): a pair over it is flagged identically in
every form (and in the oracle); all other counts are exact, and the forms'
exact match totals and flags must agree request by request.

Phases: W * 4 warm-up requests (untimed; the first tunes the matcher's
launch shape), then K * 4 requests at once (burst: throughput), then K * 4
requests arriving as a Poisson process at 70 % of the batched form's burst
request rate (latency from arrival to sorted results readable on the host).
A step is 4 requests.  The work limit (default 2^18 partial embeddings per
(query, update)) keeps the pool's explosive queries (8-10 vertices through
R-MAT hubs, up to 10^11 embeddings per request) to a bounded, flagged cost.

Prints one JSON line.  `value` = the served form's exact delta-matches per
second of device time over the burst (events around each device batch;
inputs copied from host memory inside it); `e2e` = the same matches over the
burst's wall time through the C ABI (host buffers in, sorted tuples out);
`latency_ms` = served p50 / p99 in the Poisson phase; `forms` = all three.
`cpu_baseline` = the oracle's all-cores matcher on a uniform sample of the
burst's updates (each update on the graph state it sees, every live query).
--impl reference: the CPU arm -- the same oracle port on that sample (the
reference has no CPU matcher and its GPU matcher is unwired), plus the
reference's own updateHostGraph timed on request batches.
--mode step: config 2 (2^20 vertices, 2^24 edges, three 8-vertex queries,
batches of 4096), one batch per step, counts only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode serve|step]
"""
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

REQ_PER_STEP = 4
INCOMPLETE = np.uint64(1 << 63)


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# Counters of the matcher measured by ncu (one B200, --clock-control none):
# config 4 at 1/4 scale, launches 81-83 of `bench.py --scale -2 --steps 1
# --warmup 1`; config 2 at full size, the timed launch of `bench.py --mode
# step --steps 1 --warmup 1 --autotune 0` (5 blocks per SM).
C4_NCU = {"dram_bytes_per_launch": 1.672e8, "l2_bytes_per_launch": 2.385e9, "launch_ms": 1.825,
          "l2_hit": 0.620, "issue_active": 0.180}
C2_NCU = {"dram_bytes_per_launch": 4.847e8, "l2_bytes_per_launch": None, "launch_ms": 225.4,
          "l2_hit": 0.939, "issue_active": 0.395}


def l2_figures(ncu):
    """L2 side of the roofline: the ncu L2 bytes per launch over the ncu
    launch time against an L2 copy bandwidth measured here."""
    out = {"hit_rate": ncu["l2_hit"]}
    try:
        peak = measure_l2_gbs()
    except Exception as ex:  # the figure is context; the line stands without it
        peak, out["peak_error"] = None, str(ex)
    out["peak_gbs"] = peak
    if ncu.get("l2_bytes_per_launch"):
        gbs = ncu["l2_bytes_per_launch"] / (ncu["launch_ms"] / 1e3) / 1e9
        out["ncu_gbs"] = gbs
        out["frac"] = gbs / peak if peak else None
    return out


def measure_l2_gbs():
    """L2 copy bandwidth (read + write bytes per second) measured here: a
    16 MiB -> 16 MiB copy repeated, both buffers resident in the 126 MB L2,
    CUDA events around 50 copies after 10 warm ones, best of 5."""
    import torch
    a = torch.empty(4 << 20, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    a.fill_(1.0)
    for _ in range(10):
        b.copy_(a)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(50):
            b.copy_(a)
        e1.record()
        e1.synchronize()
        best = max(best, 50 * 2 * a.numel() * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def combine_over_ranks(dev_ms, wall_ms, matches, device):
    """Whole-job figures of a replicated run: the slowest rank's times and the
    matches of all ranks (one all-reduce each; every rank calls it)."""
    import torch
    t = torch.tensor([dev_ms, wall_ms, float(matches)], dtype=torch.float64, device=device)
    mx = t.clone()
    torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
    sm = t.clone()
    torch.distributed.all_reduce(sm, op=torch.distributed.ReduceOp.SUM)
    return float(mx[0]), float(mx[1]), int(sm[2])


def summarize(lat_ms, matches, updates, span_s):
    lat = np.sort(np.asarray(lat_ms, dtype=np.float64))
    return {"p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "matches_per_sec": matches / span_s if span_s > 0 else 0.0,
            "updates_per_sec": updates / span_s if span_s > 0 else 0.0, "span_s": span_s,
            "matches": int(matches)}


# ---------------------------------------------------------------------------
# the serving comparison (config 4)
# ---------------------------------------------------------------------------
def churn_schedule(n_req, n_initial, n_pool, every=4, seed=4):
    """events[k]: the control requests that arrive with request k, in order:
    ("reg", pool index) or ("ret", index of an initial query).  Alternates
    registration and retirement; each initial query retires at most once, so
    every form can name it by the id it got at the start."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(n_initial)
    events, j, r = [[] for _ in range(n_req)], 0, 0
    for k in range(every - 1, n_req, every):
        if j % 2 == 0:
            events[k].append(("reg", int(rng.integers(n_pool))))
        elif r < n_initial - 1:
            events[k].append(("ret", int(order[r])))
            r += 1
        j += 1
    return events


def exact_matches(counts):
    c = np.asarray(counts, dtype=np.uint64)
    ok = (c & INCOMPLETE) == 0
    return int(c[ok].sum()), int((~ok).sum())


class FormRun:
    """Per-request outcomes of one form."""

    def __init__(self, n):
        self.matches = np.zeros(n, np.int64)
        self.flagged = np.zeros(n, np.int64)
        self.lat = np.zeros(n)
        self.dev_ms = np.zeros(n)  # this request's share of its device batch
        self.signs = [None] * n
        self.merged = np.ones(n)
        self.d2h = np.zeros(n, np.int64)

    def record(self, k, r, t):
        m, f = exact_matches(r.counts)
        self.matches[k], self.flagged[k] = m, f
        self.signs[k] = r.signs
        self.lat[k] = t["total_ms"]
        self.merged[k] = t["merged_requests"]
        self.dev_ms[k] = t["device_ms"] / max(t["merged_requests"], 1)
        self.d2h[k] = r.tuples.nbytes + r.counts.nbytes + r.signs.nbytes


def run_sync(e, reqs, arrivals, events, pool, initial_ids, base_k, out):
    """One request at a time in arrival order (batched and plain forms);
    control requests are applied before the request they arrive with."""
    t0 = time.perf_counter()
    for j, b in enumerate(reqs):
        k = base_k + j
        now = time.perf_counter() - t0
        if now < arrivals[j]:
            time.sleep(arrivals[j] - now)
        for kind, x in events[k]:
            if kind == "reg":
                e.register(pool[x])
            else:
                e.retire(initial_ids[x])
        bid = e.submit(b)
        t = e.timing(bid)
        r = e.results(bid)
        t = dict(t)
        t["total_ms"] = (time.perf_counter() - t0 - arrivals[j]) * 1e3
        out.record(k, r, t)
    return time.perf_counter() - t0


def run_served(e, reqs, arrivals, events, pool, initial_ids, base_k, out):
    """Requests (and control requests) submitted on their arrival times from
    a submitter thread; results read in order as they become final."""
    bids = [None] * len(reqs)
    err = []
    t0 = time.perf_counter()

    def submitter():
        try:
            for j, b in enumerate(reqs):
                now = time.perf_counter() - t0
                if now < arrivals[j]:
                    time.sleep(arrivals[j] - now)
                for kind, x in events[base_k + j]:
                    if kind == "reg":
                        e.register_async(pool[x])
                    else:
                        e.retire_async(initial_ids[x])
                bids[j] = e.submit(b)
        except Exception as ex:  # surfaced after the reader is done
            err.append(ex)

    th = threading.Thread(target=submitter)
    th.start()
    for j in range(len(reqs)):
        while bids[j] is None:
            if err:
                raise err[0]
            time.sleep(0.0002)
        t = e.timing(bids[j])
        r = e.results(bids[j])
        out.record(base_k + j, r, t)
    th.join()
    if err:
        raise err[0]
    return time.perf_counter() - t0


def restore(e, reqs, runs_signs, initial):
    """Puts the initial graph and query set back: the inverse of every
    effective update, newest first, applied without matching; then every
    query retired and the initial ones registered again (same ids)."""
    inv = []
    for b, s in zip(reversed(reqs), reversed(runs_signs)):
        eff = np.nonzero(s)[0][::-1]
        if len(eff):
            u = b[eff].copy()
            u[:, 0] = 1 - u[:, 0]
            inv.append(u)
    if inv:
        allinv = np.concatenate(inv)
        for i in range(0, len(allinv), 1 << 20):
            e.apply_graph(allinv[i:i + (1 << 20)])
    for qid in e.live_queries():
        e.retire(qid)
    ids = [e.register(q) for q in initial]
    return ids


def run_serve(args, rank=0, world=1):
    import torch

    import dsm_b200 as d
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    W, K = args.warmup * REQ_PER_STEP, args.steps * REQ_PER_STEP
    n_req = W + 2 * K
    t0 = time.time()
    w = d.Workload(4, scale_log2=args.scale, num_batches=n_req)
    gen_s = time.time() - t0
    reqs = list(w.batches())[:n_req]
    pool = w.queries
    initial = pool[:args.queries]
    events = churn_schedule(n_req, len(initial), len(pool))
    print(f"[bench] config 4: {w.nv} vertices, {len(w.edges)} edges, {len(pool)} pool queries "
          f"({min(q.nv for q in pool)}-{max(q.nv for q in pool)} vertices), {n_req} requests "
          f"(median {int(np.median([len(r) for r in reqs]))} updates), generated in {gen_s:.0f} s",
          file=sys.stderr, flush=True)
    e = d.Engine(dev)
    e.set_option(d.OPT_LIST, 1)
    e.set_option(d.OPT_FILTER, args.filter)
    if args.pack >= 0:
        e.set_option(d.OPT_PACK_MAX, args.pack)
    if args.merge >= 0:
        e.set_option(d.OPT_MERGE_MAX, args.merge)
    e.set_option(d.OPT_WORK_LIMIT, args.work_limit)
    e.set_option(d.OPT_QUERY_LIST_LIMIT, args.query_list_limit)
    t0 = time.time()
    e.load_graph_edges(w.nv, w.labels, w.edges)
    load_s = time.time() - t0
    ids = [e.register(q) for q in initial]
    print(f"[bench] graph loaded in {load_s:.0f} s; {e.stats()['device_bytes_in_use'] / 2**30:.1f} GiB on the device",
          file=sys.stderr, flush=True)

    runs, spans, stats = {}, {}, {}
    arrivals_burst = np.zeros(K)
    order = ["batched", "served", "plain"]
    rate = None
    sampler = ClockSampler(dev)
    for fi, form in enumerate(order):
        run = FormRun(n_req)
        e.set_option(d.OPT_PLAIN, int(form == "plain"))
        e.set_option(d.OPT_GRAPH, int(form == "served"))
        if fi == 0 and args.autotune:
            e.set_option(d.OPT_AUTOTUNE, 1)
        s0 = e.stats()
        if form == "served":
            e.serve_start(args.serve_merge)
            runner = run_served
        else:
            runner = run_sync
        runner(e, reqs[:W], np.zeros(W), events, pool, ids, 0, run)
        torch.cuda.synchronize()
        s1 = e.stats()
        if fi == 0:
            sampler.start()
        torch.cuda.synchronize()
        span_b = runner(e, reqs[W:W + K], arrivals_burst, events, pool, ids, W, run)
        torch.cuda.synchronize()
        s2 = e.stats()
        if rate is None:
            rate = args.load * K / span_b
            rng = np.random.default_rng(4)
            arrivals_p = np.cumsum(rng.exponential(1.0 / rate, K))
        span_p = runner(e, reqs[W + K:], arrivals_p, events, pool, ids, W + K, run)
        torch.cuda.synchronize()
        s3 = e.stats()
        if form == "served":
            e.serve_stop()
        spans[form] = (span_b, span_p)
        stats[form] = (s1, s2, s3)
        runs[form] = run
        print(f"[bench] {form}: burst {span_b:.2f} s, poisson {span_p:.2f} s, "
              f"exact matches {int(run.matches[W:].sum())}, flagged {int(run.flagged[W:].sum())}",
              file=sys.stderr, flush=True)
        if fi < len(order) - 1:
            again = restore(e, reqs, run.signs, initial)
            assert again == ids, "the initial queries came back with other ids"
    clocks = sampler.stop()
    tuned = {k: e.get_option(getattr(d, "OPT_" + k.upper()))
             for k in ("warps_per_sm", "split_min", "donate_depth", "pack_max", "merge_max", "bfs_levels")}

    # the forms must agree request by request
    ref = runs["batched"]
    for form in order[1:]:
        assert np.array_equal(runs[form].matches, ref.matches), f"{form}: exact matches differ from batched"
        assert np.array_equal(runs[form].flagged, ref.flagged), f"{form}: over-limit flags differ from batched"

    def form_summary(form):
        run, (span_b, span_p) = runs[form], spans[form]
        s1, s2, s3 = stats[form]
        mb = int(run.matches[W:W + K].sum())
        ub = int(sum(len(r) for r in reqs[W:W + K]))
        dev_ms = float(run.dev_ms[W:W + K].sum())
        burst = summarize(run.lat[W:W + K], mb, ub, span_b)
        pois = summarize(run.lat[W + K:], int(run.matches[W + K:].sum()), int(sum(len(r) for r in reqs[W + K:])),
                         span_p)
        return {"burst": burst, "poisson": pois,
                "device_matches_per_sec": mb / (dev_ms / 1e3) if dev_ms > 0 else 0.0,
                "device_updates_per_sec": ub / (dev_ms / 1e3) if dev_ms > 0 else 0.0,
                "device_ms_burst": dev_ms,
                "flagged_pairs": int(run.flagged[W:].sum()),
                "kernel_launches_burst": int(s2["kernel_launches"] - s1["kernel_launches"]),
                "mean_requests_per_device_batch": float(np.mean(run.merged[W:W + K])),
                "donations": int(s2["donations"] - s1["donations"]), "steals": int(s2["steals"] - s1["steals"]),
                "alg_bytes_burst": int(s2["alg_bytes"] - s1["alg_bytes"]),
                "graph_instantiations": int(s3["graph_instantiations"] - s1["graph_instantiations"]),
                "graph_captures": int(s3["graph_captures"] - s1["graph_captures"]),
                "compactions": int(s3["compactions"])}

    forms = {f: form_summary(f) for f in order}
    sv = forms["served"]
    mb = sv["burst"]["matches"]
    h2d = int(sum(r.nbytes for r in reqs[W:W + K]) / args.steps)
    d2h = int(runs["served"].d2h[W:W + K].sum() / args.steps)
    peak, peak_kind = _peaks()
    s1, s2, _ = stats["served"]
    match_ms = float(runs["served"].dev_ms[W:W + K].sum())
    alg = sv["alg_bytes_burst"]
    line = {
        "metric": "served_delta_matches_per_sec",
        "value": sv["device_matches_per_sec"],
        "unit": "matches/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": sv["device_ms_burst"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded R-MAT graph, random-walk queries, generated request stream)",
        "config": {"workload": f"config4: R-MAT(0.57,0.19,0.19) |V|=2^{24 + args.scale}, |E|=2^{28 + args.scale}, "
                               f"32 uniform labels, {len(initial)} initial queries of a 64-query pool (4-10 "
                               f"vertices), churn every 4th request, lognormal requests (median 512, cap 65536), "
                               f"60% inserts",
                   "step": f"{REQ_PER_STEP} requests", "listing": True, "work_limit": args.work_limit,
                   "query_list_limit": args.query_list_limit, "poisson_load": args.load,
                   "poisson_rate_per_s": rate, "parallelism": f"replicas x{world}", "filter": args.filter,
                   "tuned": tuned,
                   "l2": "inputs (2^28-edge graph, ~5 GB of runs) far larger than L2"},
        "updates_per_sec": sv["device_updates_per_sec"],
        "latency_ms": {"p50": sv["poisson"]["p50_ms"], "p99": sv["poisson"]["p99_ms"]},
        "matches": mb,
        "e2e": {"value": sv["burst"]["matches_per_sec"], "unit": "matches/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "updates_per_sec": sv["burst"]["updates_per_sec"]},
        "forms": forms,
        "served_vs_plain": {
            "burst_matches_per_sec": sv["burst"]["matches_per_sec"] / max(forms["plain"]["burst"]["matches_per_sec"],
                                                                          1e-9),
            "p99_ratio": (forms["plain"]["poisson"]["p99_ms"] or 0) / max(sv["poisson"]["p99_ms"] or 1e-9, 1e-9)},
        "gpu_launches": sv["kernel_launches_burst"],
        "roofline": {"bound": "hbm", "kernel": "k_match", "achieved": alg / 1e9 / (match_ms / 1e3) if match_ms else 0,
                     "peak": peak, "unit": "GB/s", "peak_source": peak_kind,
                     # ncu, this workload at 1/4 scale (same request sizes): DRAM
                     # read + write, L2 bytes and issue activity per k_match launch
                     "traffic": C4_NCU["dram_bytes_per_launch"],
                     "traffic_note": "ncu dram__bytes read+write per k_match launch, mean of 3 launches of this "
                                     "workload at 1/4 scale (same request sizes)",
                     "l2": l2_figures(C4_NCU),
                     "issue_active": C4_NCU["issue_active"],
                     "note": "algorithmic bytes of the matcher over the served device time of the burst; the "
                             "matcher waits on dependent L2 loads (issue_active), HBM is not the binding bound"},
        "clocks": clocks,
        "gen_seconds": gen_s,
        "load_seconds": load_s,
    }
    line["roofline"]["frac"] = line["roofline"]["achieved"] / peak
    e.close()
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(w, reqs, W, K, initial, pool, events, args.cpu_s, args.work_limit)
    return line


# ---------------------------------------------------------------------------
# CPU: the oracle port on a uniform sample
# ---------------------------------------------------------------------------
def cpu_sample(w, reqs, W, K, initial, pool, events, budget_s, work_limit, threads=None):
    """The oracle's all-cores matcher on updates sampled uniformly (fixed
    seed) from the burst's requests, each counted for every live query on the
    graph state it sees, until about budget_s seconds of matching; the rest
    of the stream only moves the oracle's graph."""
    from oracle import oracle as orc
    threads = threads or (os.cpu_count() or 1)
    q0 = initial[0]
    st = orc.Stream(w.nv, w.labels, w.edges, q0.labels, q0.offsets, q0.nbrs)
    st.set_work_limit(work_limit)
    live = list(range(len(initial)))  # pool indices of live queries (initial = pool[:n])
    init_live = {i: i for i in range(len(initial))}
    rng = np.random.default_rng(7)
    n_burst = sum(len(r) for r in reqs[W:W + K])
    per_update = max(1, n_burst // 256)
    secs, matches, probes, sampled = 0.0, 0, 0, 0
    for k, b in enumerate(reqs[:W + K]):
        for kind, x in events[k]:
            if kind == "reg":
                live.append(x)
            else:
                live.remove(init_live[x])
        if k < W or secs >= budget_s:
            st.apply_graph(b)
            continue
        pick = np.nonzero(rng.random(len(b)) < 1.0 / per_update)[0]
        prev = 0
        for i in pick:
            st.apply_graph(b[prev:i])
            prev = int(i)
            op, a, c = (int(v) for v in b[i][:3])
            for qi in live:
                q = pool[qi]
                st.set_query(q.labels, q.offsets, q.nbrs)
                t = time.perf_counter()
                cnt = st.probe(op, a, c, threads)
                secs += time.perf_counter() - t
                probes += 1
                if not (cnt >> 63):
                    matches += cnt
            sampled += 1
        st.apply_graph(b[prev:])
    return {"value": matches / secs if secs > 0 else 0.0, "unit": "matches/s", "cores": threads, "kind": "port",
            "sample": f"{sampled} updates sampled uniformly from the burst's requests (1 in {per_update}), each "
                      f"counted for every live query ({probes} counts) on the graph state it sees, "
                      f"{threads} threads, work limit {work_limit}", "seconds": secs}


def reference_update_host_graph(w, reqs, n_calls, budget_s):
    """The reference's own updateHostGraph (cpuGraph.cpp:521-607, compiled
    from its sources into oracle/_ref/libref.so) on request batches of the
    same stream: updates per second of its host path.  None when the library
    was not built."""
    import ctypes as C
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    if not os.path.exists(lib_path):
        return None
    lib = C.CDLL(lib_path)
    u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    lib.ref_graph_new.restype = C.c_void_p
    lib.ref_graph_new.argtypes = [C.c_uint32, u32p, C.c_uint64, u32p]
    lib.ref_graph_update.argtypes = [C.c_void_p, C.c_uint32, u32p]
    lib.ref_graph_free.argtypes = [C.c_void_p]
    h = lib.ref_graph_new(w.nv, w.labels, len(w.edges), np.ascontiguousarray(w.edges.reshape(-1)))
    secs, ups, calls = 0.0, 0, 0
    try:
        for b in reqs[:n_calls]:
            t = time.perf_counter()
            lib.ref_graph_update(h, len(b), np.ascontiguousarray(b.reshape(-1)))
            secs += time.perf_counter() - t
            ups += len(b)
            calls += 1
            if secs > budget_s:
                break
    finally:
        lib.ref_graph_free(h)
    return {"updates_per_sec": ups / secs if secs > 0 else 0.0, "calls": calls, "updates": ups, "seconds": secs,
            "cores": 1, "kind": "reference",
            "sample": f"the first {calls} requests, one updateHostGraph call each (rebuilds the whole CSR)"}


def run_reference(args, rank):
    """The CPU arm of the serving comparison: the oracle port on a uniform
    sample of the same burst (each step: the sample's share), plus the
    reference's own updateHostGraph on the same requests.  The inputs come
    from the engine's generator compiled into the oracle library; the engine
    library is not loaded."""
    if rank != 0:
        return None
    from oracle import oracle as orc
    W, K = args.warmup * REQ_PER_STEP, args.steps * REQ_PER_STEP
    w = orc.Workload(4, scale_log2=args.scale, num_batches=W + 2 * K)
    reqs = list(w.batches())[:W + 2 * K]
    initial = w.queries[:args.queries]
    events = churn_schedule(W + 2 * K, len(initial), len(w.queries))
    cb = cpu_sample(w, reqs, W, K, initial, w.queries, events, args.ref_s, args.work_limit)
    v = cb["value"]
    line = {"impl": "reference", "metric": "served_delta_matches_per_sec", "value": v, "unit": "matches/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["seconds"] / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (the GPU arm's seeded inputs)",
            "config": {"workload": "config4 (as the GPU arm)", "form": "CPU, per update, all host threads"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "matches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_host:
        # updateHostGraph rebuilds the whole CSR through a std::set per vertex
        # (about 20 GB of host memory at 2^28 edges): timed on the same stream
        # at 1/16 scale
        ws = orc.Workload(4, scale_log2=args.scale - 4, num_batches=8)
        rh = reference_update_host_graph(ws, list(ws.batches()), 8, args.ref_host_s)
        if rh is not None:
            rh["sample"] += f"; config-4 stream at 1/16 scale (|V|=2^{20 + args.scale}, |E|=2^{24 + args.scale})"
        line["reference_update_host_graph"] = rh
    return line


# ---------------------------------------------------------------------------
# --mode step: config 2, one 4096-update batch per step (counts)
# ---------------------------------------------------------------------------
def step_workload(args, nq, bsz):
    sc = args.scale
    if args.config == 2:
        return (f"config2: Chung-Lu gamma=2.1, |V|=2^{20 + sc}, |E|=2^{24 + sc}, 16 Zipf(1.2) labels, "
                f"three 8-vertex queries, batches of {bsz} (50/50)")
    if args.config == 3:
        return (f"config3: the config-2 graph (|V|=2^{20 + sc}), {nq} queries of 4-12 vertices in one launch, "
                f"batches of {bsz}")
    if args.config == 5:
        return (f"config5: R-MAT(0.70,0.12,0.12) |V|=2^{22 + sc}, |E|=2^{27 + sc}, 8 uniform labels, "
                f"{nq} twelve-vertex cyclic queries (two triangles + a 4-cycle), batches of {bsz} (80% deletes)")
    return f"config{args.config} at scale 2^{sc}, {nq} queries, batches of {bsz}"


def run_step(args, rank, world):
    import torch

    import dsm_b200 as d
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    t0 = time.time()
    w = d.Workload(args.config, scale_log2=args.scale, num_batches=args.steps + args.warmup)
    gen_s = time.time() - t0
    batches = list(w.batches())
    if args.batch:
        batches = [b[:args.batch] for b in batches]
    queries = w.queries[:args.queries] if args.config != 2 else w.queries
    e = d.Engine(dev)
    e.set_option(d.OPT_LIST, 0)
    if args.step_work_limit:
        e.set_option(d.OPT_WORK_LIMIT, args.step_work_limit)
    e.set_option(d.OPT_FILTER, args.filter)
    if args.pack >= 0:
        e.set_option(d.OPT_PACK_MAX, args.pack)
    if args.merge >= 0:
        e.set_option(d.OPT_MERGE_MAX, args.merge)
    if args.autotune and args.warmup > 0:
        e.set_option(d.OPT_AUTOTUNE, 1)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    for q in queries:
        e.register(q)
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")  # 256 MiB > L2
    print(f"[bench] config {args.config}: {w.nv} vertices, {len(w.edges)} edges, {len(queries)} queries, "
          f"batches of {len(batches[0])}, generated in {gen_s:.0f} s", file=sys.stderr, flush=True)
    for k, b in enumerate(batches[:args.warmup]):
        t = time.perf_counter()
        e.run_batch(b)
        print(f"[bench] warm-up batch {k}: {time.perf_counter() - t:.2f} s", file=sys.stderr, flush=True)
    sampler = ClockSampler(dev)
    if rank == 0:
        sampler.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    rows, flagged = [], 0
    for b in batches[args.warmup:args.warmup + args.steps]:
        flush.zero_()
        torch.cuda.synchronize()
        s0 = e.stats()
        tw = time.perf_counter()
        r = e.run_batch(b)
        wall = (time.perf_counter() - tw) * 1e3
        s1 = e.stats()
        c = r.counts
        exact = int(c[(c & np.uint64(1 << 63)) == 0].sum())
        flagged += int(((c & np.uint64(1 << 63)) != 0).sum())
        rows.append((s1["last_batch_ms"], wall, s1["last_match_ms"], exact,
                     s1["alg_bytes"] - s0["alg_bytes"], s1["kernel_launches"] - s0["kernel_launches"],
                     s1["donations"] - s0["donations"], s1["steals"] - s0["steals"]))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop() if rank == 0 else None
    R = np.array(rows, dtype=np.float64)
    dev_ms, wall_ms, match_ms = R[:, 0].sum(), R[:, 1].sum(), R[:, 2].sum()
    matches = int(R[:, 3].sum())
    if world > 1:
        dev_ms, wall_ms, matches = combine_over_ranks(dev_ms, wall_ms, matches, "cuda")
    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    alg = float(R[:, 4].sum())
    achieved = alg / 1e9 / (match_ms / 1e3) if match_ms > 0 else 0.0
    upd = sum(len(b) for b in batches[args.warmup:args.warmup + args.steps]) * world
    line = {"metric": "delta_matches_per_sec", "value": matches / (dev_ms / 1e3), "unit": "matches/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu graph, random-walk queries, generated update stream)",
            "config": {"workload": step_workload(args, len(queries), len(batches[0])),
                       "flagged_pairs": flagged, "work_limit": args.step_work_limit,
                       "listing": False, "parallelism": f"replicas x{world}",
                       "l2": "256 MiB buffer written between timed batches",
                       "filter": args.filter,
                       "tuned": {k: e.get_option(getattr(d, "OPT_" + k.upper()))
                                 for k in ("warps_per_sm", "split_min", "donate_depth", "pack_max", "merge_max", "bfs_levels")}},
            "updates_per_sec": upd / (dev_ms / 1e3), "matches": matches,
            "latency_ms": {"p50": float(np.percentile(R[:, 1], 50)), "p99": float(np.percentile(R[:, 1], 99))},
            "e2e": {"value": matches / (wall_ms / 1e3), "unit": "matches/s",
                    "h2d_bytes_per_step": int(np.mean([b.nbytes for b in batches[args.warmup:]])),
                    "d2h_bytes_per_step": int(len(queries) * len(batches[-1]) * 8 + len(batches[-1]))},
            "gpu_launches": int(R[:, 5].sum()), "donations": int(R[:, 6].sum()), "steals": int(R[:, 7].sum()),
            "roofline": {"bound": "hbm", "kernel": "k_match", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": C2_NCU["dram_bytes_per_launch"] if args.config == 2 and args.scale == 0 else None,
                         "traffic_note": "ncu dram__bytes read+write of one k_match launch on this workload",
                         "l2": l2_figures(C2_NCU) if args.config == 2 and args.scale == 0 else None,
                         "issue_active": C2_NCU["issue_active"] if args.config == 2 and args.scale == 0 else None},
            "clocks": clocks, "gen_seconds": gen_s}
    e.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="serve", choices=["serve", "step"])
    ap.add_argument("--config", type=int, default=2, choices=[2, 3, 5], help="--mode step: the workload")
    ap.add_argument("--batch", type=int, default=0, help="--mode step: updates per batch (0: the config's)")
    ap.add_argument("--step-work-limit", type=int, default=0, help="--mode step: DSM_OPT_WORK_LIMIT (0: none)")
    ap.add_argument("--scale", type=int, default=0, help="log2 shrink of the graph (0 = config size)")
    ap.add_argument("--queries", type=int, default=64, help="queries registered at the start (of the 64-query pool)")
    ap.add_argument("--work-limit", type=int, default=1 << 18,
                    help="partial embeddings one (query, update) search may generate")
    ap.add_argument("--query-list-limit", type=int, default=1 << 22,
                    help="tuples one query may list per device batch")
    ap.add_argument("--load", type=float, default=0.7, help="Poisson rate / batched burst rate")
    ap.add_argument("--serve-merge", type=int, default=0)
    ap.add_argument("--autotune", type=int, default=1)
    ap.add_argument("--filter", type=int, default=0, help="DSM_OPT_FILTER (0 labels only, 1 LDF+NLF, 2 cluster encoding)")
    ap.add_argument("--pack", type=int, default=-1, help="DSM_OPT_PACK_MAX before tuning (-1: engine default)")
    ap.add_argument("--merge", type=int, default=-1, help="DSM_OPT_MERGE_MAX before tuning (-1: engine default)")
    ap.add_argument("--cpu-s", type=float, default=15.0, help="seconds of CPU matching for cpu_baseline")
    ap.add_argument("--ref-s", type=float, default=60.0, help="reference arm: seconds of CPU matching")
    ap.add_argument("--ref-host-s", type=float, default=60.0, help="reference arm: seconds of updateHostGraph")
    ap.add_argument("--no-ref-host", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        # CPU arm: rank 0 alone runs; other ranks exit without work
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    pg = False
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = True
    try:
        if args.mode == "step":
            line = run_step(args, rank, world)
        else:
            line = run_serve(args, rank, world)
            if world > 1:  # replicas: the slowest rank's time, everyone's matches
                import torch
                dm, wm, mt = combine_over_ranks(line["forms"]["served"]["device_ms_burst"],
                                                line["forms"]["served"]["burst"]["span_s"] * 1e3,
                                                line["matches"], "cuda")
                line["value"] = mt / (dm / 1e3)
                line["e2e"]["value"] = mt / (wm / 1e3)
                if rank != 0:
                    line = None
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
