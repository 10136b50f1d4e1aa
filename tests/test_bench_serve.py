"""Host logic of bench.py's serving comparison, on a stand-in engine that
honours the same call contract (submit / timing / results, asynchronous
registration and retirement, admission).  No GPU."""
import os
import sys
import threading
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class StandIn:
    def __init__(self, live):
        self.lock = threading.Lock()
        self.live = set(live)
        self.sizes, self.tickets = {}, {}
        self.next_bid, self.next_ticket, self.next_qid = 1, 1, 100
        self.retired = []

    def submit(self, b):
        with self.lock:
            bid = self.next_bid
            self.next_bid += 1
            self.sizes[bid] = len(b)
            return bid

    def timing(self, bid):
        return {"total_ms": 1.0 + bid % 3}

    def results(self, bid):
        n = self.sizes.pop(bid)
        return SimpleNamespace(counts=np.full((1, n), 2, np.uint64), num_updates=n)

    def register_async(self, q):
        with self.lock:
            t = self.next_ticket
            self.next_ticket += 1
            self.tickets[t] = self.next_qid
            self.live.add(self.next_qid)
            self.next_qid += 1
            return t

    def retire_async(self, qid):
        with self.lock:
            assert qid in self.live, "retired a query that is not live"
            self.live.remove(qid)
            self.retired.append(qid)
            return 0

    def admission(self, t, timeout_ms):
        return self.tickets[t]

    def stats(self):
        return {"live_queries": len(self.live)}


def test_churn_phase_accounting():
    e = StandIn(range(6))
    n = 40
    out = bench.run_churn(e, np.linspace(0.0, 0.04, n), [np.zeros((5, 4), np.uint32)] * n, list(range(6)), ["q"])
    assert out["registrations"] + out["retirements"] == n // 4
    assert out["retirements"] > 0 and out["registrations"] > 0
    assert out["matches"] == 2 * 5 * n and out["updates_per_sec"] > 0
    assert out["live_queries_at_end"] == 6 + out["registrations"] - out["retirements"]
    assert out["admission_wait_ms"]["p50"] is not None
    assert not e.sizes  # every batch's results were read


def test_summarize():
    s = bench.summarize([1.0, 2.0, 3.0, 100.0], 50, 10, 2.0)
    assert s["p50_ms"] == 2.5 and s["matches_per_sec"] == 25.0 and s["updates_per_sec"] == 5.0
