"""Host logic of bench.py's serving comparison on stand-in engines that honour
the engine's call contract (submit / timing / results, registration and
retirement, graph-only apply), and its CPU sample on a tiny workload.  No GPU."""
import os
import sys
import threading
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class StandIn:
    """A 'graph' of undirected edges; a batch reports sign +1 / -1 for each
    effective insert / delete (0 for a no-op) and count 2 per live query."""

    def __init__(self, edges, nq):
        self.lock = threading.Lock()
        self.edges = {tuple(sorted(map(int, e))) for e in edges}
        self.live = list(range(nq))
        self.next_bid, self.pending = 1, {}
        self.calls = []

    def _apply(self, b):
        signs = np.zeros(len(b), np.int8)
        for i, (op, a, c, _) in enumerate(b):
            k = tuple(sorted((int(a), int(c))))
            if a == c:
                continue
            if op == 1 and k not in self.edges:
                self.edges.add(k)
                signs[i] = 1
            elif op == 0 and k in self.edges:
                self.edges.remove(k)
                signs[i] = -1
        return signs

    def submit(self, b):
        with self.lock:
            signs = self._apply(b)
            bid = self.next_bid
            self.next_bid += 1
            counts = np.full((len(self.live), len(b)), 2, np.uint64)
            if len(b):
                counts[0, 0] |= np.uint64(1 << 63)  # one flagged pair per batch
            self.pending[bid] = SimpleNamespace(counts=counts, signs=signs, num_updates=len(b),
                                                tuples=np.zeros(0, np.uint32))
            return bid

    def timing(self, bid):
        return {"total_ms": 1.0, "device_ms": 2.0, "merged_requests": 1}

    def results(self, bid):
        return self.pending.pop(bid)

    def register(self, q):
        with self.lock:
            qid = min(set(range(len(self.live) + 1)) - set(self.live))
            self.live.append(qid)
            self.live.sort()
            return qid

    register_async = register

    def retire(self, qid):
        with self.lock:
            self.live.remove(qid)

    retire_async = retire

    def live_queries(self):
        return list(self.live)

    def apply_graph(self, u):
        self._apply(u)


def _stream(seed=1, n=30, size=20, nv=40):
    rng = np.random.default_rng(seed)
    edges = rng.integers(0, nv, (60, 2))
    reqs = []
    for _ in range(n):
        b = np.zeros((size, 4), np.uint32)
        b[:, 0] = rng.random(size) < 0.6
        b[:, 1:3] = rng.integers(0, nv, (size, 2))
        reqs.append(b)
    return edges, reqs


def test_churn_schedule():
    ev = bench.churn_schedule(100, 8, 64)
    kinds = [e[0][0] for e in ev if e]
    assert kinds[:4] == ["reg", "ret", "reg", "ret"] and kinds.count("reg") == 13
    rets = [e[0][1] for e in ev if e and e[0][0] == "ret"]
    assert len(set(rets)) == len(rets) and len(rets) <= 7  # each initial query retires at most once
    assert ev == bench.churn_schedule(100, 8, 64)  # deterministic


def test_forms_and_restore():
    """A sync run and a served run of the same requests record the same
    per-request outcomes; restore() puts the initial graph and queries back."""
    edges, reqs = _stream()
    events = bench.churn_schedule(len(reqs), 6, 10)
    pool = ["q"] * 10
    e = StandIn(edges, 6)
    start = set(e.edges)
    ids = list(range(6))
    a = bench.FormRun(len(reqs))
    bench.run_sync(e, reqs, np.zeros(len(reqs)), events, pool, ids, 0, a)
    again = bench.restore(e, reqs, a.signs, ["q"] * 6)
    assert e.edges == start and again == ids
    b = bench.FormRun(len(reqs))
    bench.run_served(e, reqs, np.linspace(0, 0.01, len(reqs)), events, pool, ids, 0, b)
    assert np.array_equal(a.matches, b.matches) and np.array_equal(a.flagged, b.flagged)
    assert (a.flagged == 1).all()
    assert all(np.array_equal(x, y) for x, y in zip(a.signs, b.signs))


def test_cpu_sample_tiny():
    import dsm_b200 as d
    w = d.Workload(4, scale_log2=-12, num_batches=12)
    reqs = list(w.batches())
    events = bench.churn_schedule(len(reqs), 4, len(w.queries))
    out = bench.cpu_sample(w, reqs, 2, 5, w.queries[:4], w.queries, events, 2.0, 1 << 20, threads=2)
    assert out["kind"] == "port" and out["cores"] == 2 and out["seconds"] > 0


def test_summarize():
    s = bench.summarize([1.0, 2.0, 3.0, 100.0], 50, 10, 2.0)
    assert s["p50_ms"] == 2.5 and s["matches_per_sec"] == 25.0 and s["updates_per_sec"] == 5.0


def test_step_workload_names_and_l2_figures_without_gpu():
    """The step mode names each configuration by what it is; the L2 side of
    the roofline degrades to no peak (and no fraction) where the copy probe
    cannot run, instead of failing the line."""
    args = SimpleNamespace(config=2, scale=0)
    assert "config2" in bench.step_workload(args, 3, 4096) and "4096" in bench.step_workload(args, 3, 4096)
    args = SimpleNamespace(config=5, scale=-4)
    name = bench.step_workload(args, 64, 65536)
    assert "config5" in name and "2^18" in name and "twelve-vertex" in name
    import torch
    if torch.cuda.is_available():
        return
    out = bench.l2_figures(bench.C4_NCU)
    assert out["peak_gbs"] is None and out["frac"] is None
    assert out["ncu_gbs"] > 0 and 0 < out["hit_rate"] < 1
    out2 = bench.l2_figures(bench.C2_NCU)  # no L2 byte count: hit rate only
    assert "ncu_gbs" not in out2
