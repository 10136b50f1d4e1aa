"""Parity of the CUDA engine (through the C ABI) with the CPU oracle: every
update's canonically sorted embedding set must be identical.

Sizes: the oracle lists ~15M embeddings/s on one core, while config 2's
queries reach 10^9 embeddings per batch even at 1/64 of the graph, so the
oracle runs with a work budget per slice of 64 updates and the comparison
covers every update it could afford (tests.helpers); the engine always runs
whole batches and the graphs are compared in full."""
import json
import os

import numpy as np
import pytest

import dsm_b200 as d
from tests.helpers import compare_batch, oracle_apply, oracle_stream, run_stream, workload

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fresh(nv, labels, edges, queries, **opts):
    """A new engine with the graph loaded and the queries registered."""
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
    single-update batches (3276 re-inserts, 1000 deletes), graph checked
    every 500 batches and at the end."""
    w = workload(1)
    q = w.queries[0]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=500)
    assert total > 0 and checked == len(w.updates)
    off, nb = e.export_graph()
    ooff, onb = st.export()
    assert np.array_equal(off, ooff) and np.array_equal(nb, onb)
    e.close()


def test_c1_as_large_batches():
    """The same stream cut into batches of 512: sequential semantics inside a
    batch must give the same per-update sets as one update per batch."""
    w = workload(1)
    q = w.queries[0]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    ups = w.updates
    run_stream(e, [qid], [st], [ups[i:i + 512] for i in range(0, len(ups), 512)], check_graph_every=1)
    e.close()


@pytest.mark.parametrize("qi", [0, 1, 2])
def test_c2_scaled_counts(qi):
    """Config 2 shape (Chung-Lu, Zipf labels, 8-vertex tree / cycle / dense
    queries) at 2^14 vertices, two batches of 4096 mixed updates, count mode:
    exact per-update counts wherever the oracle's budget reaches, and the
    whole graph after every batch."""
    w = workload(2, scale_log2=-6, num_batches=2)
    q = w.queries[qi]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q], OPT_LIST=0)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, listed=False,
                                limit=150_000)
    assert checked >= 1024, checked
    e.close()


@pytest.mark.parametrize("qi", [0, 1, 2])
def test_c2_scaled_listing(qi):
    """Same workload, listed: every affordable update's sorted embedding set
    in the first batch of 4096."""
    w = workload(2, scale_log2=-6, num_batches=1)
    q = w.queries[qi]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, limit=50_000)
    assert checked >= 512, checked
    e.close()


@pytest.mark.parametrize("k", [0, 1])
def test_c4_thirty_two_labels(k):
    """Config 4 shape (R-MAT, 32 uniform labels: the last label slot is in
    use) at 2^16 vertices; the first two pool queries that carry label 31.
    Listed, two lognormal-size batches."""
    w = workload(4, scale_log2=-8, num_batches=2)
    q = [q for q in w.queries if 31 in q.labels.tolist()][k]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, limit=100_000)
    assert checked >= 64, checked
    e.close()


def test_labels_beyond_the_last_slot():
    """Data labels 29..34: labels >= 31 share the last slot of the
    label-major runs, and a query vertex with label 31 must match only data
    vertices whose label is exactly 31 (about 600 embeddings per query over
    2500 updates)."""
    rng = np.random.default_rng(7)
    nv = 1000
    labels = rng.integers(29, 35, nv).astype(np.uint32)
    edges = set()
    while len(edges) < 20000:
        a, b = (int(x) for x in rng.integers(0, nv, 2))
        if a != b:
            edges.add((min(a, b), max(a, b)))
    edges = np.array(sorted(edges), np.uint32)
    keep = np.ones(len(edges), bool)
    keep[rng.choice(len(edges), 1500, replace=False)] = False
    init, held = edges[keep], edges[~keep]
    ups = np.array([[1, a, b, 0] for a, b in held] + [[0, a, b, 0] for a, b in init[:1000]], np.uint32)
    ups = ups[rng.permutation(len(ups))]
    for ql in ([31, 31, 30, 29], [31, 29, 31, 31]):
        q = d.Query.from_edges(ql, [(0, 1), (1, 2), (0, 2), (2, 3)])
        e, (qid,) = _fresh(nv, labels, init, [q])
        st = oracle_stream(nv, labels, init, q)
        total, _ = run_stream(e, [qid], [st], [ups[:1200], ups[1200:]], check_graph_every=1)
        assert total > 500
        e.close()


def test_autotuned_batch_equals_oracle():
    """DSM_OPT_AUTOTUNE: the first batch times every candidate launch setting
    on its own union graph and keeps the fastest; its results and the next
    batch's (run with the tuned setting) equal the oracle's."""
    w = workload(2, scale_log2=-6, num_batches=2)
    q = w.queries[2]
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q], OPT_LIST=0, OPT_AUTOTUNE=1)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, listed=False,
                                limit=150_000)
    assert checked >= 1024
    s = e.stats()
    assert s["tune_runs"] >= 2 and s["tune_best_ms"] > 0
    assert e.get_option(d.OPT_AUTOTUNE) == 0
    assert e.get_option(d.OPT_SPLIT_MIN) in (64, 128, 512)
    assert e.get_option(d.OPT_DONATE_DEPTH) in (1, 2)
    assert e.get_option(d.OPT_WARPS_PER_SM) % 8 == 0
    e.close()


def test_graph_replay_equals_eager():
    """DSM_OPT_GRAPH: the batch segments run as CUDA graphs (captured, then
    updated in place while their topology repeats); listed results and the
    graph equal the eager engine's, batch by batch."""
    w = workload(1)
    q = w.queries[0]
    eager, (qa,) = _fresh(w.nv, w.labels, w.edges, [q])
    graph, (qb,) = _fresh(w.nv, w.labels, w.edges, [q], OPT_GRAPH=1)
    ups = w.updates
    for i in range(0, len(ups), 128):
        ra, rb = eager.run_batch(ups[i:i + 128]), graph.run_batch(ups[i:i + 128])
        assert np.array_equal(ra.signs, rb.signs) and np.array_equal(ra.counts, rb.counts)
        assert np.array_equal(ra.tuples, rb.tuples)
    for x, y in zip(eager.export_graph(), graph.export_graph()):
        assert np.array_equal(x, y)
    s = graph.stats()
    nb = (len(ups) + 127) // 128
    assert s["graph_launches"] == 2 * nb
    # captured once per segment (plus a re-capture when a buffer grew), then
    # replayed for batches of any size
    assert s["graph_instantiations"] <= 2, s
    assert s["graph_captures"] <= 6, s
    eager.close()
    graph.close()


def test_graph_replay_varying_sizes():
    """Batches of very different sizes replay the same two executable graphs:
    the kernels read the sizes from the device header."""
    w = workload(1)
    q = w.queries[0]
    eager, (qa,) = _fresh(w.nv, w.labels, w.edges, [q])
    graph, (qb,) = _fresh(w.nv, w.labels, w.edges, [q], OPT_GRAPH=1)
    sizes = [1024, 7, 300, 1, 0, 999, 64, 500, 3]
    pos = 0
    for k in sizes:
        b = w.updates[pos:pos + k]
        pos += k
        ra, rb = eager.run_batch(b), graph.run_batch(b)
        assert np.array_equal(ra.signs, rb.signs) and np.array_equal(ra.counts, rb.counts)
        assert np.array_equal(ra.tuples, rb.tuples)
    s = graph.stats()
    assert s["graph_instantiations"] <= 2, s
    assert s["graph_captures"] <= 4, s
    for x, y in zip(eager.export_graph(), graph.export_graph()):
        assert np.array_equal(x, y)
    eager.close()
    graph.close()


def test_graph_replay_with_filter_multi_query():
    """Graph replay with the cluster filter inside the captured segment, 16
    config-3 queries, against the oracle."""
    w = workload(3, scale_log2=-6, num_batches=2)
    bs = [b[:512] for b in w.batches()]
    qs = w.queries[:16]
    e, qids = _fresh(w.nv, w.labels, w.edges, qs, OPT_GRAPH=1, OPT_FILTER=2)
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs]
    total, checked = run_stream(e, qids, streams, bs, check_graph_every=1, limit=200_000)
    assert checked >= 16 * 256
    assert e.stats()["graph_launches"] == 4
    e.close()


def test_listing_limit_downgrades_to_counts():
    w = workload(1, scale_log2=-2)
    b = np.concatenate(list(w.batches())[:400])
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [w.queries[0]], OPT_LIST_LIMIT=64)
    r = e.run_batch(b)
    st = oracle_stream(w.nv, w.labels, w.edges, w.queries[0])
    s, c, _ = st.apply(b, listed=False)
    if c.sum() * (w.queries[0].nv + 1) * 4 > 64:
        assert not r.listed
    assert np.array_equal(r.counts[0], c)
    e.close()


def test_multi_query_batched():
    """Config 3 shape scaled: 32 queries of 4-12 vertices in one launch; each
    query's listed results equal the oracle's for that query alone."""
    w = workload(3, scale_log2=-6, num_batches=2)
    bs = [b[:1024] for b in w.batches()]
    qs = w.queries[:32]
    e, qids = _fresh(w.nv, w.labels, w.edges, qs)
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs]
    total, checked = run_stream(e, qids, streams, bs, check_graph_every=1, limit=200_000)
    assert checked >= 32 * 512, checked
    e.close()


def test_multi_query_counts_all_256():
    """All 256 config-3 queries (scaled graph) in one launch, count mode."""
    w = workload(3, scale_log2=-6, num_batches=1)
    b = next(w.batches())[:256]
    e, qids = _fresh(w.nv, w.labels, w.edges, w.queries, OPT_LIST=0)
    assert len(qids) == 256
    r = e.run_batch(b)
    checked = 0
    for qid, q in zip(qids, w.queries):  # one oracle graph at a time
        s, c, _, v = oracle_apply(oracle_stream(w.nv, w.labels, w.edges, q), b, False, limit=500_000)
        checked += compare_batch(r, qid, s, c, None, v, tag=f"query {qid}")
    assert checked >= 256 * 128, checked
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
    eset = edges
    edges = np.array(sorted(edges), np.uint32)
    q = d.Query.from_edges([0, 0, 1, 1], [(0, 1), (1, 2), (2, 0), (2, 3)])
    e, (qid,) = _fresh(nv, labels, edges, [q])
    st = oracle_stream(nv, labels, edges, q)
    a, b = int(edges[0][0]), int(edges[0][1])
    x, y = 1, 2
    while (min(x, y), max(x, y)) in eset:
        y += 1
    z = 8 if (7, 8) not in eset else 9
    ups = [[1, x, y, 0], [1, y, x, 0], [0, x, y, 0], [1, x, y, 0],  # dup insert, delete, re-insert
           [0, a, b, 0], [1, a, b, 0], [0, b, a, 0],                # delete, re-insert, delete
           [0, 7, z, 0],                                            # delete of an absent edge
           [1, 5, 5, 0], [0, 5, 5, 0]]                              # self loops
    ups += [[int(rng.integers(0, 2)), int(rng.integers(0, nv)), int(rng.integers(0, nv)), 0] for _ in range(400)]
    run_stream(e, [qid], [st], [np.array(ups, np.uint32)], check_graph_every=1)
    run_stream(e, [qid], [st], [np.zeros((0, 4), np.uint32)], check_graph_every=1)
    e.close()


def test_one_edge_query_and_count_mode():
    w = workload(1, scale_log2=-2)
    q = d.Query.from_edges([0, 1], [(0, 1)])
    big = np.concatenate(list(w.batches())[:300])
    e, (qid, _) = _fresh(w.nv, w.labels, w.edges, [q, w.queries[0]])
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    run_stream(e, [qid], [st], [big])
    e.close()
    # count-only mode gives the same counts
    e1, _ = _fresh(w.nv, w.labels, w.edges, [w.queries[0]], OPT_LIST=0)
    e2, _ = _fresh(w.nv, w.labels, w.edges, [w.queries[0]])
    r1, r2 = e1.run_batch(big), e2.run_batch(big)
    assert not r1.listed and r2.listed
    assert np.array_equal(r1.counts, r2.counts)
    e1.close()
    e2.close()


def test_result_regrow_and_no_donation_agree():
    """A tiny result capacity forces the overflow-and-rerun path; donation
    off gives the same sets."""
    w = workload(2, scale_log2=-6, num_batches=1)
    q = w.queries[2]
    b = next(w.batches())[:1024]
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    e, (qid,) = _fresh(w.nv, w.labels, w.edges, [q], OPT_RESULT_CAP=16, OPT_DONATE=0)
    run_stream(e, [qid], [st], [b], limit=300_000)
    assert e.stats()["result_regrows"] >= 1
    e.close()


def test_retire_and_register_between_batches():
    w = workload(3, scale_log2=-6, num_batches=3)
    bs = [b[:512] for b in w.batches()]
    qs = w.queries[:6]
    e, qids = _fresh(w.nv, w.labels, w.edges, qs[:4])
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs[:4]]
    run_stream(e, qids, streams, bs[:1], limit=200_000)
    e.retire(qids[1])
    run_stream(e, [qids[0]] + qids[2:], [streams[0]] + streams[2:], bs[1:2], limit=200_000)
    qn = e.register(qs[5])
    stn = oracle_stream(w.nv, w.labels, _edges_of(e), qs[5])
    run_stream(e, [qids[0], qn], [streams[0], stn], bs[2:3], limit=200_000)
    e.close()


def _edges_of(e):
    """Undirected edge list of the engine's current graph."""
    off, nb = e.export_graph()
    src = np.repeat(np.arange(len(off) - 1, dtype=np.uint32), np.diff(off))
    m = src < nb
    return np.stack([src[m], nb[m]], axis=1)
