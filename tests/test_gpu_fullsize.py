"""Parity on the work the benchmark times, at full size.

The budgeted oracle of the other parity tests skips the heaviest updates,
which are the ones that dominate a timed batch.  Here the engine runs whole
batches in count mode on full-size graphs, and for each query the oracle's
all-cores matcher recounts the heaviest updates (up to a ceiling it finishes
in seconds) and some random ones, each on exactly the graph state that update
sees (the oracle's graph is advanced to just before it; `probe` counts the
update without applying it).  Counts must be equal.

- config 2 at full size: 2^20 vertices, 2^24 edges, the three 8-vertex
  queries, one 4096-update batch;
- config 3: 256 queries of 4-12 vertices on the full-size graph, one
  512-update slice, all queries in one launch (every 8th query recounted;
  each search bounded by a work limit of 2^22, flags checked alike);
- config 4 at full size (2^24 vertices, 2^28 edges): the benchmark's first
  request against all 64 queries under its work limit;
- config 5 at 1/16 scale (2^18 vertices, 2^23 edges, hubs above 10^4): 64
  twelve-vertex cyclic queries, one 65,536-update batch, 80 % deletions
  (every 4th query recounted).
"""
import numpy as np
import pytest

import dsm_b200 as d
from tests.helpers import workload
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _engine_counts(w, queries, batch, work_limit=0):
    e = d.Engine(0)
    e.set_option(d.OPT_LIST, 0)
    e.set_option(d.OPT_WORK_LIMIT, work_limit)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qids = [e.register(q) for q in queries]
    r = e.run_batch(batch)
    counts = np.stack([r.counts[r.query_index(q)] for q in qids])
    signs = r.signs.copy()
    st = e.stats()
    e.close()
    return counts, signs, st


def _pick(counts, heavy, ceiling, n_random, rng, top_ceiling=None):
    """Per query: its `heavy` largest exact counts at or below the ceiling
    (the first query's largest may reach top_ceiling) and n_random others
    (searches flagged over a work limit included)."""
    picks = []
    for k, c in enumerate(counts):
        exact = np.where((c & d.INCOMPLETE) == 0, c, 0).astype(np.float64)
        idx = np.argsort(-exact, kind="stable")
        cap = top_ceiling if (top_ceiling and k == 0) else ceiling
        chosen = [int(i) for i in idx if 0 < exact[i] <= cap][:heavy]
        rest = np.setdiff1d(np.arange(len(c)), chosen)
        chosen += [int(i) for i in rng.choice(rest, min(n_random, len(rest)), replace=False)]
        picks.append(sorted(set(chosen)))
    return picks


def _every(picks, step):
    """Keep the picks of every step-th query (the rest stay unchecked)."""
    return [p if k % step == 0 else [] for k, p in enumerate(picks)]


def _oracle_check(w, queries, batch, counts, picks, work_limit=0):
    """Oracle counts of the picked updates on the graph state each one sees
    (with the engine's work limit: a flagged search must be flagged alike,
    an exact one equal)."""
    q0 = queries[0]
    st = orc.Stream(w.nv, w.labels, w.edges, q0.labels, q0.offsets, q0.nbrs)
    st.set_work_limit(work_limit)
    by_update = {}
    for k, p in enumerate(picks):
        for i in p:
            by_update.setdefault(i, []).append(k)
    prev, compared, heaviest = 0, 0, 0
    for i in sorted(by_update):
        st.apply_graph(batch[prev:i])
        prev = i
        op, a, b = (int(x) for x in batch[i][:3])
        for k in by_update[i]:
            q = queries[k]
            st.set_query(q.labels, q.offsets, q.nbrs)
            got = st.probe(op, a, b)
            mine = int(counts[k][i])
            if (got >> 63) or (mine >> 63):
                assert (got >> 63) == (mine >> 63), f"query {k} update {i}: flags differ"
            else:
                assert got == mine, f"query {k} update {i}: engine {mine} oracle {got}"
                heaviest = max(heaviest, int(got))
            compared += 1
    return compared, heaviest


def test_c2_full_size_heaviest_updates():
    w = workload(2, num_batches=1)
    batch = next(w.batches())
    counts, signs, st = _engine_counts(w, w.queries, batch)
    assert counts.sum() > 10 ** 8
    picks = _pick(counts, heavy=4, ceiling=3 * 10 ** 8, n_random=6, rng=np.random.default_rng(2),
                  top_ceiling=2 * 10 ** 9)
    compared, heaviest = _oracle_check(w, w.queries, batch, counts, picks)
    assert compared >= 3 * 8
    assert heaviest > 10 ** 8, heaviest


def test_c3_full_size_256_queries_one_launch():
    w = workload(3, num_batches=1)
    batch = next(w.batches())[:512]
    lim = 1 << 22  # 256 queries of up to 12 vertices: some searches are unbounded otherwise
    counts, signs, st = _engine_counts(w, w.queries, batch, work_limit=lim)
    assert counts.shape[0] == 256
    # all 256 queries run in the launch; every 8th is recounted by the oracle
    picks = _every(_pick(counts, heavy=2, ceiling=2 * 10 ** 7, n_random=1, rng=np.random.default_rng(3)), 8)
    compared, heaviest = _oracle_check(w, w.queries, batch, counts, picks, work_limit=lim)
    assert compared >= 32  # each checked query: its heaviest exact counts (if any) and a random one


def test_c5_skew_scaled_twelve_vertex_queries():
    w = workload(5, scale_log2=-4, num_batches=1)
    deg = np.bincount(w.edges.reshape(-1), minlength=w.nv)
    assert deg.max() > 10 ** 4  # hub vertices
    batch = next(w.batches())
    assert len(batch) == 65536 and (batch[:, 0] == 0).mean() > 0.75
    lim = 1 << 22
    counts, signs, st = _engine_counts(w, w.queries, batch, work_limit=lim)
    picks = _every(_pick(counts, heavy=1, ceiling=5 * 10 ** 7, n_random=1, rng=np.random.default_rng(5)), 4)
    compared, heaviest = _oracle_check(w, w.queries, batch, counts, picks, work_limit=lim)
    assert compared >= 16
    assert st["donations"] > 0


def test_c4_full_size_first_request_64_queries():
    """The benchmark's own workload at full size (R-MAT 2^24 vertices, 2^28
    edges, 32 labels): its first request (211 updates) against all 64
    queries of 4-10 vertices in one launch, each search bounded by the
    benchmark's work limit (2^18).  For every query the oracle recounts its
    two heaviest exact updates and a random one (flags compared alike)."""
    lim = 1 << 18
    w = workload(4, num_batches=1)
    batch = next(w.batches())
    counts, signs, st = _engine_counts(w, w.queries, batch, work_limit=lim)
    assert counts.shape[0] == 64
    picks = _pick(counts, heavy=2, ceiling=10 ** 9, n_random=1, rng=np.random.default_rng(4))
    compared, heaviest = _oracle_check(w, w.queries, batch, counts, picks, work_limit=lim)
    assert compared >= 64
    assert heaviest > 0
