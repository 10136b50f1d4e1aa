"""Parity of the CUDA engine (through the C ABI) with the CPU oracle: every
update's canonically sorted embedding set must be identical."""
import json
import os

import numpy as np
import pytest

import dsm_b200 as d
from oracle import oracle as orc
from tests.helpers import compare_batch, oracle_stream, run_stream

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def eng():
    e = d.Engine(0)
    yield e
    e.close()


def _fresh(e, nv, labels, edges, queries, **opts):
    """Loads a graph and registers queries on a new engine."""
    e = d.Engine(0)
    for k, v in opts.items():
        e.set_option(getattr(d, k), v)
    e.load_graph_edges(nv, labels, edges)
    qids = [e.register(q) for q in queries]
    return e, qids


def test_kat_reference_fixture():
    kat = json.load(open(os.path.join(GOLD, "kat.json")))
    q = d.TextGraph(os.path.join(GOLD, kat["query"]), True).query()
    g = d.TextGraph(os.path.join(GOLD, kat["data"]), False)
    e = d.Engine(0)
    e.load_graph_csr(g.offsets, g.nbrs, g.labels)
    qid = e.register(q)
    r = e.run_batch(g.updates)
    assert r.signs.tolist() == kat["signs"]
    assert r.tuples_of(qid, 0).tolist() == kat["positive"][0]
    e.close()


def test_c1_stream_one_update_per_batch():
    """Config 1: R-MAT 4096 vertices, one 5-vertex one-cycle query, 4276
    single-update batches (3276 re-inserts, 1000 deletes)."""
    w = d.Workload(1)
    q = w.queries[0]
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=500)
    assert total > 0
    off, nb = e.export_graph()
    ooff, onb = st.export()
    assert np.array_equal(off, ooff) and np.array_equal(nb, onb)
    e.close()


@pytest.mark.parametrize("qi", [0, 1, 2])
def test_c2_scaled_counts(qi):
    """Config 2 shape (Chung-Lu, Zipf labels, 8-vertex tree / cycle / dense
    queries), scaled to 2^14 vertices, batches of 4096 mixed updates: exact
    per-update counts (count mode) and the graph after every batch."""
    w = d.Workload(2, scale_log2=-6, num_batches=2)
    q = w.queries[qi]
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [q], OPT_LIST=0)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, listed=False)
    e.close()


@pytest.mark.parametrize("qi", [0, 1, 2])
def test_c2_scaled_listing(qi):
    """Same workload, listed: every update's sorted embedding set, on the
    longest prefix of the first batch whose listing stays below 2M tuples."""
    w = d.Workload(2, scale_log2=-6, num_batches=1)
    q = w.queries[qi]
    b = next(w.batches())
    n = len(b)
    while n > 16:
        c = oracle_stream(w.nv, w.labels, w.edges, q).apply(b[:n], listed=False)[1]
        if c.sum() <= 2_000_000:
            break
        n //= 4
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    run_stream(e, [qid], [st], [b[:n], b[n:n + 64]], check_graph_every=1)
    e.close()


def test_listing_limit_downgrades_to_counts():
    w = d.Workload(1, scale_log2=-2)
    b = np.concatenate(list(w.batches())[:400])
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [w.queries[0]], OPT_LIST_LIMIT=64)
    r = e.run_batch(b)
    st = oracle_stream(w.nv, w.labels, w.edges, w.queries[0])
    s, c, _ = st.apply(b, listed=False)
    if c.sum() * (w.queries[0].nv + 1) * 4 > 64:
        assert not r.listed
    assert np.array_equal(r.counts[0], c)
    e.close()


def _listable(w, queries, batches, limit):
    """Queries whose oracle count over `batches` stays below `limit`."""
    out = []
    for q in queries:
        st = oracle_stream(w.nv, w.labels, w.edges, q)
        tot = 0
        for b in batches:
            tot += int(st.apply(b, listed=False)[1].sum())
            if tot > limit:
                break
        if tot <= limit:
            out.append(q)
    return out


def test_multi_query_batched():
    """Config 3 shape scaled: up to 24 queries of 4-12 vertices in one launch;
    each query's results equal the oracle's for that query alone."""
    w = d.Workload(3, scale_log2=-6, num_batches=2)
    bs = list(w.batches())
    qs = _listable(w, w.queries[:64], bs, 300_000)[:24]
    assert len(qs) >= 8
    e, qids = _fresh(None, w.nv, w.labels, w.edges, qs)
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs]
    run_stream(e, qids, streams, bs)
    e.close()


def test_multi_query_counts_all_256():
    """All 256 config-3 queries (scaled graph) in one launch, count mode: each
    query's per-update counts equal the oracle's."""
    w = d.Workload(3, scale_log2=-6, num_batches=1)
    b = next(w.batches())[:256]
    e, qids = _fresh(None, w.nv, w.labels, w.edges, w.queries, OPT_LIST=0)
    r = e.run_batch(b)
    assert len(qids) == 256
    for qid, q in list(zip(qids, w.queries))[::4]:
        s, c, _ = oracle_stream(w.nv, w.labels, w.edges, q).apply(b, listed=False)
        assert np.array_equal(r.counts[r.query_index(qid)], c), f"query {qid}"
    e.close()


def test_batch_edge_cases():
    """Within one batch: duplicate inserts, insert then delete, delete then
    re-insert, deletes of absent edges, self loops, an empty batch."""
    rng = np.random.default_rng(5)
    nv = 300
    labels = rng.integers(0, 2, nv).astype(np.uint32)
    edges = set()
    while len(edges) < 1500:
        a, b = rng.integers(0, nv, 2)
        if a != b:
            edges.add((int(min(a, b)), int(max(a, b))))
    edges = np.array(sorted(edges), np.uint32)
    q = d.Query.from_edges([0, 0, 1, 1], [(0, 1), (1, 2), (2, 0), (2, 3)])
    e, (qid,) = _fresh(None, nv, labels, edges, [q])
    st = oracle_stream(nv, labels, edges, q)
    a, b = int(edges[0][0]), int(edges[0][1])
    x, y = 1, 2
    while (min(x, y), max(x, y)) in set(map(tuple, edges.tolist())):
        y += 1
    ups = [[1, x, y, 0], [1, y, x, 0], [0, x, y, 0], [1, x, y, 0],  # dup insert, delete, re-insert
           [0, a, b, 0], [1, a, b, 0], [0, b, a, 0],                # delete, re-insert, delete
           [0, 7, 8 if (7, 8) not in set(map(tuple, edges.tolist())) else 9, 0],
           [1, 5, 5, 0], [0, 5, 5, 0]]                               # self loops
    ups += [[int(rng.integers(0, 2)), int(rng.integers(0, nv)), int(rng.integers(0, nv)), 0] for _ in range(400)]
    run_stream(e, [qid], [st], [np.array(ups, np.uint32)], check_graph_every=1)
    run_stream(e, [qid], [st], [np.zeros((0, 4), np.uint32)], check_graph_every=1)
    e.close()


def test_one_edge_query_and_count_mode():
    w = d.Workload(1, scale_log2=-2)
    q = d.Query.from_edges([0, 1], [(0, 1)])
    ups = list(w.batches())
    big = np.concatenate(ups[:300])
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [q, w.queries[0]])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    run_stream(e, [qid], [st], [big])
    e.close()
    # count-only mode gives the same counts
    e1, q1 = _fresh(None, w.nv, w.labels, w.edges, [w.queries[0]], OPT_LIST=0)
    e2, q2 = _fresh(None, w.nv, w.labels, w.edges, [w.queries[0]])
    r1, r2 = e1.run_batch(big), e2.run_batch(big)
    assert not r1.listed and r2.listed
    assert np.array_equal(r1.counts, r2.counts)
    e1.close()
    e2.close()


def test_result_regrow_and_no_donation_agree():
    """A tiny result capacity forces the overflow-and-rerun path; donation
    off gives the same sets."""
    w = d.Workload(2, scale_log2=-6, num_batches=2)
    q = w.queries[2]
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    e, (qid,) = _fresh(None, w.nv, w.labels, w.edges, [q], OPT_RESULT_CAP=16, OPT_DONATE=0)
    run_stream(e, [qid], [st], list(w.batches()))
    assert e.stats()["result_regrows"] >= 1
    e.close()


def test_retire_and_register_between_batches():
    w = d.Workload(3, scale_log2=-6, num_batches=3)
    bs = [b[:1024] for b in w.batches()]
    qs = _listable(w, w.queries[:40], bs, 200_000)[:6]
    e, qids = _fresh(None, w.nv, w.labels, w.edges, qs[:4])
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs[:4]]
    run_stream(e, qids, streams, bs[:1])
    e.retire(qids[1])
    for st in streams[1:2]:
        st.apply(bs[1], listed=False)
    run_stream(e, [qids[0]] + qids[2:], [streams[0]] + streams[2:], bs[1:2])
    qn = e.register(qs[5])
    off, nb = e.export_graph()
    edges = np.array([(v, int(x)) for v in range(w.nv) for x in nb[off[v]:off[v + 1]] if v < x], np.uint32)
    stn = oracle_stream(w.nv, w.labels, edges, qs[5])
    run_stream(e, [qids[0], qn], [streams[0], stn], bs[2:3])
    e.close()
