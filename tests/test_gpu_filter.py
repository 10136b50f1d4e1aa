"""The GPU cluster-encoding candidate filter against the oracle's restatement
of the reference filter (filter.cu): per-u candidate bitmaps and the LDF+NLF
masks must be identical; with the filter pruning the matcher, every update's
embeddings must still equal the oracle's (which matches without a filter)."""
import numpy as np
import pytest

import dsm_b200 as d
from oracle import oracle as orc
from tests.helpers import oracle_stream, run_stream, workload

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
    w = workload(cfg, scale_log2=-6 if cfg > 1 else 0, num_batches=1)
    queries = w.queries[:48]
    ops = _filter_case(w.nv, w.labels, w.edges, queries)
    assert ops >= len(queries)  # every query ran at least one op


def test_filter_random_queries_with_merges_and_combines():
    """Random trees and cyclic queries of 5-12 vertices exercise the merge
    and combine ops of the clustering plan."""
    rng = np.random.default_rng(3)
    w = workload(1)
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
    w = workload(1)
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
    w = workload(3, scale_log2=-6, num_batches=2)
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
    w = workload(2, scale_log2=-6, num_batches=2)
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


def _inc_pair(w, queries, mode=2, **opts):
    engines = []
    for inc in (1, 0):
        e = d.Engine(0)
        e.set_option(d.OPT_FILTER, mode)
        e.set_option(d.OPT_FILTER_INCREMENTAL, inc)
        for k, v in opts.items():
            e.set_option(getattr(d, k), v)
        e.load_graph_edges(w.nv, w.labels, w.edges)
        engines.append((e, [e.register(q) for q in queries]))
    return engines


def _same_state(inc, full, queries, nv, tag):
    """Resident filter state of the incremental engine == the full one's;
    returns the runs that were incremental and their vertex counts."""
    (ei, qi), (ef, qf) = inc, full
    runs = []
    for a, b, q in zip(qi, qf, queries):
        bi, vi, (fi, ni) = ei.filter_state(a, q.nv, nv)
        bf, vf, (ff, nf) = ef.filter_state(b, q.nv, nv)
        assert ff and nf == nv, tag
        assert np.array_equal(vi, vf), f"{tag} query {a}: LDF+NLF masks differ at {np.nonzero(vi != vf)[0][:8]}"
        assert np.array_equal(bi, bf), f"{tag} query {a}: bitmaps differ (u {np.nonzero((bi != bf).any(1))[0]})"
        if not fi:
            runs.append(ni)
    return runs


@pytest.mark.parametrize("cfg,scale,nqs,bsz,nb", [(1, 0, 1, 32, 10), (2, -4, 3, 8, 10), (3, -6, 16, 64, 6),
                                                  (4, -10, 8, 16, 8)])
def test_incremental_filter_equals_full(cfg, scale, nqs, bsz, nb):
    """DSM_OPT_FILTER_INCREMENTAL: after every batch the resident bitmaps and
    LDF+NLF masks of the incremental filter (region of the batch's and the
    previous batch's endpoints, validity replay outside it) equal those of a
    full recompute on the same union graph; the matches are identical; later
    batches ran incrementally on regions smaller than the graph."""
    w = workload(cfg, scale_log2=scale, num_batches=1)
    qs = w.queries[:nqs]
    inc, full = _inc_pair(w, qs)
    ups = next(w.batches())
    region_runs = []
    for k in range(nb):
        b = ups[k * bsz:(k + 1) * bsz]
        ri, rf = inc[0].run_batch(b), full[0].run_batch(b)
        assert np.array_equal(ri.counts, rf.counts) and np.array_equal(ri.tuples, rf.tuples)
        region_runs += _same_state(inc, full, qs, w.nv, f"batch {k}")
    assert len(region_runs) >= (nb - 1) * len(qs) // 2, region_runs
    assert min(region_runs) < w.nv
    for e, _ in (inc, full):
        e.close()


def test_incremental_filter_ldf_only_and_graph_changes():
    """Mode 1 (LDF+NLF, a region of the endpoints alone), a graph-only apply
    between batches (the next run recomputes every vertex), and CUDA-graph
    replay: the state still equals a full recompute after every batch."""
    w = workload(2, scale_log2=-4, num_batches=1)
    qs = w.queries[:3]
    ups = next(w.batches())
    for mode, opts in ((1, {}), (2, {"OPT_GRAPH": 1})):
        inc, full = _inc_pair(w, qs, mode=mode, **opts)
        fulls = 0
        for k in range(8):
            b = ups[k * 16:(k + 1) * 16]
            if k == 4:  # graph-only apply: not filtered
                for e, _ in (inc, full):
                    e.apply_graph(ups[200:232])
            ri, rf = inc[0].run_batch(b), full[0].run_batch(b)
            assert np.array_equal(ri.counts, rf.counts)
            runs = _same_state(inc, full, qs, w.nv, f"mode {mode} batch {k}")
            if k == 4:
                assert runs == [], "the run after a graph-only apply must be full"
            fulls += len(qs) - len(runs)
        assert fulls < 8 * len(qs)
        for e, _ in (inc, full):
            e.close()
