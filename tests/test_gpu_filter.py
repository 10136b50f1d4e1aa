"""The GPU cluster-encoding candidate filter against the oracle's restatement
of the reference filter (filter.cu): per-u candidate bitmaps and the LDF+NLF
masks must be identical; with the filter pruning the matcher, every update's
embeddings must still equal the oracle's (which matches without a filter)."""
import numpy as np
import pytest

import dsm_b200 as d
from oracle import oracle as orc
from tests.helpers import oracle_stream, run_stream

pytestmark = pytest.mark.gpu


def _filter_case(nv, labels, edges, queries):
    e = d.Engine(0)
    e.load_graph_edges(nv, labels, edges)
    qids = [e.register(q) for q in queries]
    off, nb = e.export_graph()
    checked = 0
    for qid, q in zip(qids, queries):
        bm, vc = e.filter(qid, q.nv, nv)
        obm, ovc, pos, plan = orc.cluster_filter(q.labels, q.offsets, q.nbrs, nv, labels, off, nb)
        assert np.array_equal(vc, ovc), f"query {qid}: LDF+NLF masks differ"
        assert np.array_equal(bm, obm), f"query {qid}: bitmaps differ at u {np.nonzero((bm != obm).any(1))[0]}"
        checked += len(plan)
    e.close()
    return checked


def test_filter_reference_fixture():
    import os
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    q = d.TextGraph(os.path.join(gold, "example_q_01.in"), True).query()
    g = d.TextGraph(os.path.join(gold, "example_g_01.in"), False)
    _filter_case(g.nv, g.labels, g.edges, [q])


@pytest.mark.parametrize("cfg", [1, 2, 3])
def test_filter_bitmaps_match_oracle(cfg):
    w = d.Workload(cfg, scale_log2=-6 if cfg > 1 else 0, num_batches=1)
    queries = w.queries[:48]
    ops = _filter_case(w.nv, w.labels, w.edges, queries)
    assert ops >= len(queries)  # every query ran at least one op


def test_filter_random_queries_with_merges_and_combines():
    """Random trees and cyclic queries of 5-12 vertices exercise the merge
    and combine ops of the clustering plan."""
    rng = np.random.default_rng(3)
    w = d.Workload(1)
    qs = []
    for _ in range(24):
        nq = int(rng.integers(5, 13))
        edges = {(int(rng.integers(0, v)), v) for v in range(1, nq)}
        while len(edges) < nq - 1 + int(rng.integers(0, 3)):
            a, b = sorted(int(x) for x in rng.integers(0, nq, 2))
            if a != b:
                edges.add((a, b))
        qs.append(d.Query.from_edges(rng.integers(0, 4, nq), sorted(edges)))
    _filter_case(w.nv, w.labels, w.edges, qs)


@pytest.mark.parametrize("mode", [1, 2])
def test_matching_with_filter_c1(mode):
    w = d.Workload(1)
    q = w.queries[0]
    e = d.Engine(0)
    e.set_option(d.OPT_FILTER, mode)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(q)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    ups = w.updates
    run_stream(e, [qid], [st], [ups[i:i + 512] for i in range(0, len(ups), 512)], check_graph_every=1)
    e.close()


def test_matching_with_filter_multi_query():
    w = d.Workload(3, scale_log2=-6, num_batches=2)
    bs = [b[:1024] for b in w.batches()]
    qs = w.queries[:32]
    e = d.Engine(0)
    e.set_option(d.OPT_FILTER, 2)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qids = [e.register(q) for q in qs]
    streams = [oracle_stream(w.nv, w.labels, w.edges, q) for q in qs]
    total, checked = run_stream(e, qids, streams, bs, check_graph_every=1, limit=200_000)
    assert checked >= 32 * 512
    e.close()


@pytest.mark.parametrize("qi", [0, 1, 2])
def test_matching_with_filter_c2_counts(qi):
    w = d.Workload(2, scale_log2=-6, num_batches=2)
    q = w.queries[qi]
    e = d.Engine(0)
    e.set_option(d.OPT_FILTER, 2)
    e.set_option(d.OPT_LIST, 0)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(q)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    total, checked = run_stream(e, [qid], [st], list(w.batches()), check_graph_every=1, listed=False,
                                limit=150_000)
    assert checked >= 1024
    e.close()
