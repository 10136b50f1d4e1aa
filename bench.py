#!/usr/bin/env python
"""Benchmark: continuous subgraph matching on one B200 (config 2).

Workload (seeded, synthetic; the reference's dataset is not available):
Chung-Lu power-law graph (exponent 2.1), 2^20 vertices, 2^24 undirected
edges (10% withheld for re-insertion), 16 Zipf(1.2) labels; three 8-vertex
random-walk queries (tree, one cycle, 14 edges); batches of 4096 updates,
50% inserts from the withheld pool, 50% deletes of live edges.

A step is one update batch matched against the three queries, exact counts
per update (--list 1 lists and sorts the embeddings as well).  Forms:
  batched (default): one engine, all queries in one persistent launch;
  plain: one engine per query, one launch per query (the reference's
         one-query-per-process form).
The first warm-up batch autotunes the matcher's launch setting (--autotune).

Prints one JSON line.  `value` = delta-matches per second of device time
(CUDA events around each batch's device work); `e2e` = the same through the
C ABI with host buffers (host prep, H2D, matching, D2H, result assembly) on
the wall clock; `cpu_baseline` = the oracle's all-cores matcher on a prefix
of the first timed batch (counts).  --impl reference: the CPU arm (the same
oracle port, all host threads, a bounded prefix of each timed batch).
--mode serve: served vs batched vs plain on the config-4 request stream
(throughput under a burst, p50 / p99 latency under Poisson arrivals).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode step|serve]
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


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


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


def make_workload(steps, warmup, scale):
    import dsm_b200 as d
    nb = steps + warmup
    return d.Workload(2, scale_log2=scale, num_batches=nb)


def run_ours(args, rank, world):
    import torch

    import dsm_b200 as d
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    t0 = time.time()
    w = make_workload(args.steps, args.warmup, args.scale)
    gen_s = time.time() - t0
    batches = list(w.batches())
    queries = w.queries
    print(f"[bench] workload generated in {gen_s:.1f} s: {w.nv} vertices, {len(w.edges)} edges, "
          f"queries {[q.labels.tolist() for q in queries]}", file=sys.stderr, flush=True)

    def new_engine(qs):
        e = d.Engine(dev)
        e.set_option(d.OPT_LIST, args.list)
        e.set_option(d.OPT_FILTER, args.filter)
        if args.autotune and args.warmup > 0:  # the first warm-up batch picks the launch setting
            e.set_option(d.OPT_AUTOTUNE, 1)
        e.load_graph_edges(w.nv, w.labels, w.edges)
        return e, [e.register(q) for q in qs]

    if args.form == "batched":
        engines = [new_engine(queries)]
    else:
        engines = [new_engine([q]) for q in queries]
    print(f"[bench] {len(engines)} engine(s) loaded", file=sys.stderr, flush=True)
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")  # 256 MiB > L2

    def step(b):
        """One batch through every engine; device ms, wall ms, matches, stats deltas."""
        dev_ms = wall_ms = match_ms = 0.0
        matches = alg = launches = 0
        h2d = d2h = 0
        for e, qids in engines:
            s0 = e.stats()
            torch.cuda.synchronize()
            tw = time.perf_counter()
            r = e.run_batch(b)
            wall_ms += (time.perf_counter() - tw) * 1e3
            s1 = e.stats()
            dev_ms += s1["last_batch_ms"]
            match_ms += s1["last_match_ms"]
            matches += int(r.counts.sum())
            alg += s1["alg_bytes"] - s0["alg_bytes"]
            launches += s1["kernel_launches"] - s0["kernel_launches"]
            h2d += b.nbytes
            d2h += r.tuples.nbytes + r.counts.nbytes + r.signs.nbytes
            if args.verbose:
                print(f"  engine {qids}: dev {s1['last_batch_ms']:.2f} ms match {s1['last_match_ms']:.2f} ms "
                      f"upd {s1['last_update_ms']:.2f} ms filter {s1['last_filter_ms']:.2f} ms wall {(time.perf_counter() - tw) * 1e3:.1f} ms "
                      f"matches {int(r.counts.sum())} per-query {r.counts.sum(axis=1).tolist()} "
                      f"seeds {s1['seeds'] - s0['seeds']} donations {s1['donations'] - s0['donations']} "
                      f"listed {r.listed}", file=sys.stderr, flush=True)
        return dev_ms, wall_ms, match_ms, matches, alg, launches, h2d, d2h

    for b in batches[:args.warmup]:
        step(b)
    rows = []
    sampler = ClockSampler(dev)
    if rank == 0:
        sampler.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for b in batches[args.warmup:args.warmup + args.steps]:
        flush.zero_()
        torch.cuda.synchronize()
        rows.append(step(b))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop() if rank == 0 else None
    R = np.array([r[:6] for r in rows], dtype=np.float64)
    dev_ms, wall_ms, match_ms = R[:, 0].sum(), R[:, 1].sum(), R[:, 2].sum()
    matches = int(R[:, 3].sum())
    alg = float(R[:, 4].sum())
    launches = int(R[:, 5].sum())
    h2d = int(sum(r[6] for r in rows) / len(rows))
    d2h = int(sum(r[7] for r in rows) / len(rows))
    if world > 1:
        dev_ms, wall_ms, matches = combine_over_ranks(dev_ms, wall_ms, matches, "cuda")
    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    upd = sum(len(b) for b in batches[args.warmup:args.warmup + args.steps]) * world
    lat = np.sort(R[:, 1])
    achieved = alg / 1e9 / (match_ms / 1e3) if match_ms > 0 else 0.0
    line = {
        "metric": "delta_matches_per_sec",
        "value": matches / (dev_ms / 1e3) if dev_ms > 0 else 0.0,
        "unit": "matches/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded Chung-Lu graph, random-walk queries, generated update stream)",
        "config": {"workload": f"config2: Chung-Lu gamma=2.1, |V|=2^{20 + args.scale}, |E|=2^{24 + args.scale}, "
                               "16 Zipf(1.2) labels, three 8-vertex queries, batches of 4096 (50/50)",
                   "form": args.form, "listing": bool(args.list), "filter": args.filter,
                   "tuned": {k: engines[0][0].get_option(getattr(d, "OPT_" + k.upper()))
                             for k in ("warps_per_sm", "split_min", "donate_depth")}, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed batches"},
        "updates_per_sec": upd / (dev_ms / 1e3) if dev_ms > 0 else 0.0,
        "matches": matches,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "e2e": {"value": matches / (wall_ms / 1e3) if wall_ms > 0 else 0.0, "unit": "matches/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "updates_per_sec": upd / (wall_ms / 1e3) if wall_ms > 0 else 0.0},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_match", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                     "alg_bytes_per_step": alg / args.steps},
        "clocks": clocks,
        "gen_seconds": gen_s,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, batches, args.warmup)
    return line


def summarize(lat_ms, matches, updates, span_s):
    lat = np.sort(np.asarray(lat_ms))
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "matches_per_sec": matches / span_s, "updates_per_sec": updates / span_s, "span_s": span_s,
            "matches": int(matches)}


def run_churn(e, arrivals, batch_list, live, pool):
    """Poisson batches; every 4th arrival also registers a pool query or
    retires a live one (alternately, keeping at least 4 live), through
    the serving loop's queue.  Admission waits are timed per ticket."""
    import random
    rnd = random.Random(4)
    bids, tickets, lock = [], [], threading.Lock()
    counts = {"registrations": 0, "retirements": 0}
    base = time.perf_counter()

    def submitter():
        for k, (a, b) in enumerate(zip(arrivals, batch_list)):
            now = time.perf_counter() - base
            if now < a:
                time.sleep(a - now)
            if k % 4 == 3:
                with lock:
                    retire = (k // 4) % 2 == 1 and len(live) > 4
                    victim = live.pop(rnd.randrange(len(live))) if retire else None
                if retire:
                    e.retire_async(victim)
                    counts["retirements"] += 1
                else:
                    tickets.append((e.register_async(pool[(k // 4) % len(pool)]), time.perf_counter()))
                    counts["registrations"] += 1
            bids.append(e.submit(b))

    waits = []

    def admitter():  # admission outcome of each registration, in order
        k = 0
        while k < len(tickets) or th.is_alive():
            if k >= len(tickets):
                time.sleep(0.001)
                continue
            t, t_sub = tickets[k]
            qid = e.admission(t, 60_000)
            waits.append((time.perf_counter() - t_sub) * 1e3)
            if qid is not None:
                with lock:
                    live.append(qid)
            k += 1

    th = threading.Thread(target=submitter)
    th.start()
    ta = threading.Thread(target=admitter)
    ta.start()
    lat, matches, upd = [], 0, 0
    for k in range(len(batch_list)):
        while len(bids) <= k:
            time.sleep(0.0002)
        t = e.timing(bids[k])
        r = e.results(bids[k])
        lat.append(t["total_ms"])
        matches += int(r.counts.sum())
        upd += r.num_updates
    th.join()
    ta.join()
    out = summarize(lat, matches, upd, time.perf_counter() - base)
    out.update(counts)
    out["admission_wait_ms"] = {"p50": float(np.median(waits)) if waits else None,
                                "max": float(max(waits)) if waits else None}
    out["live_queries_at_end"] = e.stats()["live_queries"]
    return out


def run_serve(args):
    """Serving comparison on the config-4 stream (R-MAT, 32 uniform labels,
    lognormal batch sizes with median 512, 60% inserts): the same requests
    through three forms, each from the same initial graph.
      plain:   one engine per query, one launch per query per batch, in turn;
      batched: one engine, all queries in one launch per batch;
      served:  one engine with the serving loop (continuous batching) and
               CUDA-graph replay of each device batch.
    Phase 1 (burst): every request at t=0 -> throughput.  Phase 2 (the next
    requests): Poisson arrivals at 70% of the batched form's burst request
    rate -> p50 / p99 latency from arrival to results readable on the host.
    Phase 3 (served form only, the next requests): the same arrivals with
    query registrations and retirements through the serving loop's queue."""
    import torch

    import dsm_b200 as d
    torch.cuda.set_device(0)
    K = args.serve_requests
    scale = args.scale if args.scale else -6
    t0 = time.time()
    w = d.Workload(4, scale_log2=scale, num_batches=3 * K)
    gen_s = time.time() - t0
    reqs = list(w.batches())[:3 * K]
    burst, poisson, churn = reqs[:K], reqs[K:2 * K], reqs[2 * K:]
    # 8-10-vertex random-walk queries through the R-MAT hubs carry up to
    # 10^11 embeddings per request at this scale; the serving comparison uses
    # the pool's queries of at most 7 vertices
    qs = [q for q in w.queries if q.nv <= 7][:args.serve_queries]
    print(f"[serve] workload in {gen_s:.1f} s: {w.nv} vertices, {len(w.edges)} edges, {len(qs)} queries, "
          f"request sizes median {int(np.median([len(r) for r in reqs]))} max {max(len(r) for r in reqs)}",
          file=sys.stderr, flush=True)

    def engine(qlist, graph=False):
        e = d.Engine(0)
        e.set_option(d.OPT_LIST, args.list)
        e.set_option(d.OPT_GRAPH, int(graph))
        e.load_graph_edges(w.nv, w.labels, w.edges)
        return e, [e.register(q) for q in qlist]

    def run_sync(engines, arrivals, batch_list):
        """One request at a time, in arrival order, through every engine."""
        lat, matches, upd = [], 0, 0
        torch.cuda.synchronize()
        base = time.perf_counter()
        for a, b in zip(arrivals, batch_list):
            now = time.perf_counter() - base
            if now < a:
                time.sleep(a - now)
            for e, _ in engines:
                r = e.run_batch(b)
                matches += int(r.counts.sum())
            lat.append((time.perf_counter() - base - a) * 1e3)
            upd += len(b)
        return summarize(lat, matches, upd, time.perf_counter() - base)

    def run_served(e, arrivals, batch_list):
        bids = []
        base = time.perf_counter()

        def submitter():
            for a, b in zip(arrivals, batch_list):
                now = time.perf_counter() - base
                if now < a:
                    time.sleep(a - now)
                bids.append(e.submit(b))

        th = threading.Thread(target=submitter)
        th.start()
        lat, matches, upd, merged = [], 0, 0, []
        for k in range(len(batch_list)):
            while len(bids) <= k:
                time.sleep(0.0002)
            t = e.timing(bids[k])
            r = e.results(bids[k])
            lat.append(t["total_ms"])
            merged.append(t["merged_requests"])
            matches += int(r.counts.sum())
            upd += r.num_updates
        th.join()
        out = summarize(lat, matches, upd, time.perf_counter() - base)
        out["mean_requests_per_device_batch"] = float(np.mean(merged))
        return out

    arms = {}
    sampler = ClockSampler(0)
    sampler.start()
    # batched first: its burst rate sets the Poisson rate
    e, _ = engine(qs)
    arms["batched"] = {"burst": run_sync([(e, None)], np.zeros(K), burst)}
    rate = 0.7 * K / arms["batched"]["burst"]["span_s"]
    arrivals = np.cumsum(np.random.default_rng(4).exponential(1.0 / rate, K))
    arms["batched"]["poisson"] = run_sync([(e, None)], arrivals, poisson)
    e.close()
    print(f"[serve] batched done; Poisson rate {rate:.1f} requests/s", file=sys.stderr, flush=True)
    e, ids = engine(qs, graph=True)  # the served form replays its batch segments as CUDA graphs
    e.serve_start(args.serve_merge)
    arms["served"] = {"burst": run_served(e, np.zeros(K), burst), "poisson": run_served(e, arrivals, poisson)}
    # served only: the same arrivals with query churn (other forms would need
    # engines to come and go; the live set differs, so no cross-form check)
    pool = [q for q in w.queries if q.nv <= 7][args.serve_queries:] or qs
    arms["served"]["churn"] = run_churn(e, arrivals, churn, list(ids), pool)
    e.serve_stop()
    e.close()
    print("[serve] served done", file=sys.stderr, flush=True)
    engines = [engine([q]) for q in qs]
    arms["plain"] = {"burst": run_sync(engines, np.zeros(K), burst), "poisson": run_sync(engines, arrivals, poisson)}
    for e, _ in engines:
        e.close()
    clocks = sampler.stop()
    for k in ("batched", "served", "plain"):
        assert arms[k]["burst"]["matches"] == arms["batched"]["burst"]["matches"], "forms disagree"
        assert arms[k]["poisson"]["matches"] == arms["batched"]["poisson"]["matches"], "forms disagree"
    sv = arms["served"]["poisson"]
    return {
        "metric": "served_p99_batch_latency_ms", "value": sv["p99_ms"], "unit": "ms", "n_gpus": 1,
        "higher_is_better": False, "dtype": "u32", "data": "synthetic (seeded R-MAT graph, generated stream)",
        "config": {"workload": f"config4 stream on R-MAT(0.57,0.19,0.19) |V|=2^{24 + scale}, "
                               f"|E|=2^{28 + scale}, 32 uniform labels, {len(qs)} queries of 4-7 vertices "
                               f"(the first of the 64-query pool of 4-10 vertices with at most 7), "
                               f"lognormal request sizes (median 512), 60% inserts",
                   "requests_per_phase": K, "poisson_rate_per_s": rate, "listing": bool(args.list),
                   "max_merge_updates": args.serve_merge or 65536},
        "arms": arms, "clocks": clocks, "gen_seconds": gen_s,
    }


def _oracle_sample(streams, batch, target_s, threads):
    """Counts (all host threads) on the batch's first updates, 16 at a time,
    until target_s seconds of matching; then the rest of the batch is applied
    to the graphs without matching.  Returns (matches, seconds, updates)."""
    matches, secs, pos = 0, 0.0, 0
    while pos < len(batch) and secs < target_s:
        chunk = batch[pos:pos + 16]
        for st in streams:
            t = time.perf_counter()
            _, c, _ = st.apply(chunk, listed=False, threads=threads)
            secs += time.perf_counter() - t
            matches += int(c.sum())
        pos += len(chunk)
    for st in streams:
        st.apply_graph(batch[pos:])
    return matches, secs, pos


def _oracle_streams(w, warm):
    from oracle import oracle as orc
    streams = [orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs) for q in w.queries]
    for b in warm:  # the graph state the first timed batch sees
        for st in streams:
            st.apply_graph(b)
    return streams


def cpu_baseline(w, batches, warmup, target_s=10.0):
    """The oracle (CPU restatement of the same per-update matching, exact
    counts, all host threads) on a prefix of the first timed batch, on the
    graph state that batch sees on the GPU."""
    threads = os.cpu_count() or 1
    streams = _oracle_streams(w, batches[:warmup])
    matches, secs, n = _oracle_sample(streams, batches[warmup], target_s, threads)
    return {"value": matches / secs if secs > 0 else 0.0, "unit": "matches/s", "cores": threads, "kind": "port",
            "sample": f"first {n} updates of the first timed batch x {len(w.queries)} queries, counts, "
                      f"{threads} threads", "seconds": secs}


def run_reference(args, rank):
    """The CPU arm: each step = a bounded prefix of that step's batch (about
    args.ref_step_s seconds of matching on all host threads), counts."""
    if rank != 0:
        return None
    w = make_workload(args.steps, args.warmup, args.scale)
    batches = list(w.batches())
    threads = os.cpu_count() or 1
    streams = _oracle_streams(w, batches[:args.warmup])
    secs = matches = upd = 0
    for b in batches[args.warmup:args.warmup + args.steps]:
        m, s, n = _oracle_sample(streams, b, args.ref_step_s, threads)
        matches, secs, upd = matches + m, secs + s, upd + n
    v = matches / secs if secs > 0 else 0.0
    return {"impl": "reference", "metric": "delta_matches_per_sec", "value": v, "unit": "matches/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": {"workload": "config2 (as the GPU arm)", "form": "CPU, per update"},
            "cpu_baseline": {"value": v, "unit": "matches/s", "cores": threads, "kind": "port",
                             "sample": f"{upd} updates: a prefix of each timed batch (about {args.ref_step_s} s "
                                       f"each) x {len(w.queries)} queries, counts"},
            "e2e": {"value": v, "unit": "matches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    # config 2's tree and one-cycle queries give 10^6..10^9 embeddings per batch
    # at full size: the default measures exact counts (listing is covered by
    # the parity tests); --list 1 lists and sorts them as well
    ap.add_argument("--list", type=int, default=0)
    ap.add_argument("--filter", type=int, default=0, help="candidate filter: 0 none, 1 LDF+NLF, 2 cluster encoding")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--autotune", type=int, default=1, help="1: tune the matcher launch on the first warm-up batch")
    ap.add_argument("--scale", type=int, default=0, help="log2 shrink of the graph (0 = config size)")
    ap.add_argument("--ref-step-s", type=float, default=5.0, help="CPU arm: seconds of matching per step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="step", choices=["step", "serve"],
                    help="serve: served vs batched vs plain on the config-4 request stream")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-queries", type=int, default=16)
    ap.add_argument("--serve-merge", type=int, default=0)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.mode == "serve":
        print(json.dumps(run_serve(args)), flush=True)
        return
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
        line = run_ours(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if pg:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
