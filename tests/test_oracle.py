"""The CPU oracle pinned against the reference's fixture and against
independent checks (brute force, count identities).  No GPU."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kat():
    with open(os.path.join(GOLD, "kat.json")) as f:
        return json.load(f)


def test_kat_reference_fixture():
    kat = _kat()
    q = orc.parse(os.path.join(GOLD, kat["query"]), True)
    g = orc.parse(os.path.join(GOLD, kat["data"]), False)
    assert q["nv"] == 5 and q["ne"] == 5 and g["nv"] == 11 and g["ne"] == 13
    assert g["updates"].tolist() == kat["updates"] and g["batch_sizes"].tolist() == [1]
    s = orc.Stream(g["nv"], g["labels"], g["edges"], q["labels"], q["offsets"], q["nbrs"])
    assert s.count_all() == kat["count_before"]
    signs, counts, tuples = s.apply(g["updates"])
    assert signs.tolist() == kat["signs"]
    assert tuples[0].tolist() == kat["positive"][0]
    assert s.count_all() == kat["count_after"]


def _random_graph(rng, nv, ne, nl):
    labels = rng.integers(0, nl, nv).astype(np.uint32)
    edges = set()
    while len(edges) < ne:
        a, b = rng.integers(0, nv, 2)
        if a != b:
            edges.add((min(a, b), max(a, b)))
    return labels, np.array(sorted(edges), np.uint32)


def _csr(nv, edges):
    adj = [[] for _ in range(nv)]
    for a, b in edges:
        adj[a].append(b)
        adj[b].append(a)
    off = np.zeros(nv + 1, np.uint32)
    nb = []
    for v in range(nv):
        nb += sorted(adj[v])
        off[v + 1] = len(nb)
    return off, np.array(nb, np.uint32)


QUERIES = [
    ([0, 0, 0], [(0, 1), (1, 2), (0, 2)]),                   # triangle
    ([0, 1, 0, 1], [(0, 1), (1, 2), (2, 3)]),                 # path
    ([0, 0, 1, 1], [(0, 1), (1, 2), (2, 3), (0, 3)]),         # 4-cycle
    ([1, 0, 0, 0, 1], [(0, 1), (0, 2), (0, 3), (3, 4)]),      # tree
    ([0, 0], [(0, 1)]),                                       # one edge
]


@pytest.mark.parametrize("qi", range(len(QUERIES)))
def test_stream_matches_bruteforce(qi):
    """Per-update sets vs brute-force counts before/after each update, on
    graphs small enough to enumerate every injective map."""
    import dsm_b200 as d
    rng = np.random.default_rng(100 + qi)
    ql, qe = QUERIES[qi]
    q = d.Query.from_edges(ql, qe)
    nv = 9
    labels, edges = _random_graph(rng, nv, 16, 2)
    st = orc.Stream(nv, labels, edges, q.labels, q.offsets, q.nbrs)
    cur = set(map(tuple, edges.tolist()))

    def bf():
        off, nb = _csr(nv, sorted(cur))
        return orc.bruteforce_count(q.labels, q.offsets, q.nbrs, nv, labels, off, nb)

    before = bf()
    assert st.count_all() == before
    for step in range(40):
        a, b = (int(x) for x in rng.integers(0, nv, 2))
        op = int(rng.integers(0, 2))
        signs, counts, tuples = st.apply(np.array([[op, a, b, labels[a]]]))
        key = (min(a, b), max(a, b))
        if a == b:
            assert signs[0] == 0
            continue
        if op == 1 and key not in cur:
            cur.add(key)
            after = bf()
            assert signs[0] == 1 and after - before == counts[0]
        elif op == 0 and key in cur:
            cur.discard(key)
            after = bf()
            assert signs[0] == -1 and before - after == counts[0]
        else:
            after = before
            assert signs[0] == 0 and counts[0] == 0
        # every tuple is an embedding that uses the updated edge
        for t in tuples[0]:
            assert len(set(t.tolist())) == len(t)
            assert all(labels[t[u]] == q.labels[u] for u in range(q.nv))
            used = {(min(t[x], t[y]), max(t[x], t[y])) for x, y in qe}
            assert key in used
        assert st.count_all() == after
        before = after


def test_count_identity_c1():
    """Sum over a stream of |P| - |N| equals the change of the total count."""
    import dsm_b200 as d
    w = d.Workload(1)
    q = w.queries[0]
    st = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
    c0 = st.count_all()
    ups = w.updates[:600]
    signs, counts, _ = st.apply(ups, listed=False)
    c1 = st.count_all()
    delta = int((counts.astype(np.int64) * signs.astype(np.int64)).sum())
    assert delta == int(c1) - int(c0)


def test_parser_rejects_malformed(tmp_path):
    p = tmp_path / "bad.in"
    p.write_text("t 2 1\nv 0 0 1\nv 1 0 1\ne 0 5\n")
    with pytest.raises(ValueError):
        orc.parse(str(p), True)
    p.write_text("t 2 1\nv 1 0 1\nv 0 0 1\ne 0 1\n")
    with pytest.raises(ValueError):
        orc.parse(str(p), True)


@pytest.mark.parametrize("qi", range(len(QUERIES)))
def test_multithreaded_matcher_equals_sequential(qi):
    """The all-cores matcher (the CPU baseline) gives the sequential one's
    signs, counts and sorted tuples; apply_graph reaches the same graph."""
    rng = np.random.default_rng(11 + qi)
    labels, edges = _random_graph(rng, 60, 400, 2)
    ql, qe = QUERIES[qi]
    qoff, qnb = _csr(len(ql), qe)
    ups = []
    for _ in range(300):
        a, b = (int(x) for x in rng.integers(0, 60, 2))
        ups.append([int(rng.integers(0, 2)), a, b, 0])
    ups = np.array(ups, np.uint32)
    one = orc.Stream(60, labels, edges, np.array(ql, np.uint32), qoff, qnb)
    many = orc.Stream(60, labels, edges, np.array(ql, np.uint32), qoff, qnb)
    graph = orc.Stream(60, labels, edges, np.array(ql, np.uint32), qoff, qnb)
    s1, c1, t1 = one.apply(ups)
    s2, c2, t2 = many.apply(ups, threads=4)
    graph.apply_graph(ups)
    assert c1.sum() > 0
    assert np.array_equal(s1, s2) and np.array_equal(c1, c2)
    assert all(np.array_equal(x, y) for x, y in zip(t1, t2))
    for a, b in zip(one.export(), graph.export()):
        assert np.array_equal(a, b)


def _embeddings(labels, adj, ql, qe):
    """All embeddings by brute force (tiny graphs only)."""
    import itertools
    nq, nv = len(ql), len(labels)
    out = []
    for f in itertools.permutations(range(nv), nq):
        if all(labels[f[u]] == ql[u] for u in range(nq)) and all(f[b] in adj[f[a]] for a, b in qe):
            out.append(f)
    return out


@pytest.mark.parametrize("seed", range(12))
def test_cluster_filter_is_sound(seed):
    """The restated cluster filter (filter.cu) never drops a data vertex that
    some embedding maps a query vertex to, and the LDF+NLF masks do not
    either: the bitmaps are supersets of the true candidate sets."""
    rng = np.random.default_rng(100 + seed)
    nv = 11
    labels, edges = _random_graph(rng, nv, 30, 2)
    adj = [set() for _ in range(nv)]
    for a, b in edges:
        adj[a].add(int(b))
        adj[b].add(int(a))
    ql, qe = QUERIES[seed % len(QUERIES)]
    qoff, qnb = _csr(len(ql), qe)
    off, nb = _csr(nv, edges)
    emb = _embeddings(labels, adj, ql, qe)
    bm, vc, _, _ = orc.cluster_filter(np.array(ql, np.uint32), qoff, qnb, nv, labels, off, nb)
    for f in emb:
        for u, v in enumerate(f):
            assert (bm[u][v // 32] >> (v % 32)) & 1, f"embedding {f}: vertex {v} pruned for u{u}"
            assert (vc[v] >> u) & 1


def test_probe_and_set_query_equal_apply():
    """probe(update) on the graph before it == the count apply() reports, and
    one graph serves several queries through set_query."""
    import dsm_b200 as d  # the seeded workload generator
    w = d.Workload(3, scale_log2=-8, num_batches=1)
    ups = next(w.batches())[:200]
    qs = w.queries[:3]
    st = orc.Stream(w.nv, w.labels, w.edges, qs[0].labels, qs[0].offsets, qs[0].nbrs)
    want = []
    for q in qs:
        ref = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
        want.append(ref.apply(ups, listed=False)[1])
    for i, u in enumerate(ups):
        for k, q in enumerate(qs):
            st.set_query(q.labels, q.offsets, q.nbrs)
            assert st.probe(u[0], u[1], u[2], threads=2) == want[k][i], (i, k)
        st.apply_graph(ups[i:i + 1])


def test_oracle_workload_equals_engine_workload():
    """The CPU arms generate their inputs through the oracle library; they
    must be the engine's inputs exactly."""
    import dsm_b200 as d
    for cfg, sc in ((1, 0), (3, -8), (4, -12)):
        a, b = d.Workload(cfg, scale_log2=sc, num_batches=3), orc.Workload(cfg, scale_log2=sc, num_batches=3)
        assert a.nv == b.nv and np.array_equal(a.labels, b.labels) and np.array_equal(a.edges, b.edges)
        assert np.array_equal(a.updates, b.updates) and np.array_equal(a.batch_sizes, b.batch_sizes)
        assert len(a.queries) == len(b.queries)
        for x, y in zip(a.queries, b.queries):
            assert np.array_equal(x.labels, y.labels) and np.array_equal(x.offsets, y.offsets)
            assert np.array_equal(x.nbrs, y.nbrs)


def test_work_limit_flags_do_not_depend_on_threads():
    """The per-update search bound flags the same updates, with the same
    exact counts elsewhere, on one thread and on many."""
    import dsm_b200 as d
    w = d.Workload(3, scale_log2=-8, num_batches=1)
    ups = next(w.batches())[:300]
    INC = np.uint64(1 << 63)
    for q in w.queries[:6]:
        a = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
        full = a.apply(ups, listed=False)[1]
        a = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
        b = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
        lim = int(np.percentile(full[full > 0], 75)) if (full > 0).any() else 10
        a.set_work_limit(lim)
        b.set_work_limit(lim)
        ca = a.apply(ups, listed=False)[1]
        cb = b.apply(ups, listed=False, threads=4)[1]
        fa, fb = (ca & INC) != 0, (cb & INC) != 0
        assert np.array_equal(fa, fb)
        assert np.array_equal(ca[~fa], cb[~fb])
        assert np.array_equal(ca[~fa], full[~fa])
        # an update whose embeddings alone reach the bound is always flagged
        assert fa[full >= lim].all()
