"""The oracle's restatements of decycle (decycle.cpp:6-135) and of the BFS
matching order with backward neighbours (order.cpp:367-402, 647-676) against
the reference's own code, compiled from its sources into oracle/_ref/libref.so
by oracle/ref.mk (skipped where that library was not built).  No GPU.

The reference reads a query's neighbour lists in file order
(io.cu:181-189) and tests adjacency with a binary search over them
(is_neighbor, order.h:9-27), so with a file whose edges are not listed in
ascending (src < dst) order some backward neighbours go unseen.  The
restatement tests true adjacency; on ascending files the two agree exactly,
on other files the reference's masks are a subset of the restatement's."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref/libref.so not built")


def _lib():
    lib = C.CDLL(LIB)
    u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
    lib.ref_decycle.argtypes = [C.c_uint32, C.c_uint32, u32p, u8p, u32p]
    lib.ref_order.argtypes = [C.c_uint32, C.c_uint32, u32p, C.c_uint32, C.c_uint32, u32p, u32p]
    return lib


def _csr_file_order(nq, edges):
    """Query CSR as readGraphToCPUDynamic fills it (io.cu:181-189)."""
    deg = np.zeros(nq, np.int64)
    for a, b in edges:
        deg[a] += 1
        deg[b] += 1
    off = np.zeros(nq + 1, np.uint32)
    off[1:] = np.cumsum(deg)
    fill = off[:-1].astype(np.int64).copy()
    nb = np.zeros(int(off[-1]), np.uint32)
    for a, b in edges:
        nb[fill[a]] = b
        fill[a] += 1
        nb[fill[b]] = a
        fill[b] += 1
    return off, nb


def _random_query(rng, nq, extra):
    extra = min(extra, nq * (nq - 1) // 2 - (nq - 1))
    edges = set()
    for v in range(1, nq):
        edges.add((int(rng.integers(0, v)), v))
    while len(edges) < nq - 1 + extra:
        a, b = (int(x) for x in rng.integers(0, nq, 2))
        if a != b and (a, b) not in edges and (b, a) not in edges:
            edges.add((a, b))
    edges = [e if rng.integers(0, 2) else (e[1], e[0]) for e in sorted(edges)]
    perm = rng.permutation(nq)  # relabel so the tree root is not always 0
    edges = [(int(perm[a]), int(perm[b])) for a, b in edges]
    return [edges[i] for i in rng.permutation(len(edges))]


def _queries(ascending):
    rng = np.random.default_rng(2024)
    qs = [(5, [(0, 1), (1, 2), (2, 0), (1, 3), (3, 4)])]  # the fixture query's shape
    for _ in range(60):
        nq = int(rng.integers(3, 13))
        qs.append((nq, _random_query(rng, nq, int(rng.integers(0, nq)))))
    if ascending:  # the order a file sorted by (src, dst) with src < dst lists them in
        qs = [(nq, sorted(tuple(sorted(e)) for e in edges)) for nq, edges in qs]
    return qs


@pytest.mark.parametrize("ascending", [True, False])
@pytest.mark.parametrize("k", range(61))
def test_decycle_and_order_against_reference(k, ascending):
    lib = _lib()
    nq, edges = _queries(ascending)[k]
    flat = np.array(edges, np.uint32).reshape(-1)
    ne = len(edges)
    qoff, qnbr = _csr_file_order(nq, edges)
    # decycle: the same spanning tree and degrees
    keep = np.zeros(ne, np.uint8)
    deg = np.zeros(nq, np.uint32)
    assert lib.ref_decycle(nq, ne, flat, keep, deg) == 0
    ref_tree = {tuple(sorted(edges[e])) for e in range(ne) if keep[e]}
    toff, tnbr, tdeg = orc.decycle(qoff, qnbr)
    ours = {tuple(sorted((u, int(w)))) for u in range(nq) for w in tnbr[toff[u]:toff[u + 1]]}
    assert ours == ref_tree
    assert np.array_equal(tdeg, deg)
    # matching order and backward neighbours for every ordered query edge
    for a, b in edges:
        for u, v in ((a, b), (b, a)):
            ro = np.zeros(nq, np.uint32)
            rb = np.zeros(nq, np.uint32)
            assert lib.ref_order(nq, ne, flat, u, v, ro, rb) == 0
            oo, ob = orc.order(qoff, qnbr, u, v)
            assert np.array_equal(oo, ro), (u, v)
            if ascending:
                assert np.array_equal(ob, rb), (u, v)
            else:
                assert np.array_equal(ob & rb, rb), (u, v)  # the reference's masks miss some


def _ref_graph_lib():
    lib = C.CDLL(LIB)
    u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    lib.ref_graph_new.restype = C.c_void_p
    lib.ref_graph_new.argtypes = [C.c_uint32, u32p, C.c_uint64, u32p]
    lib.ref_graph_update.argtypes = [C.c_void_p, C.c_uint32, u32p]
    lib.ref_graph_export.restype = C.c_uint64
    lib.ref_graph_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ref_graph_free.argtypes = [C.c_void_p]
    return lib


def _ref_export(lib, h, nv):
    off = np.zeros(nv + 1, np.uint32)
    n = lib.ref_graph_export(h, off.ctypes.data, None, None)
    nb = np.zeros(max(n, 1), np.uint32)
    lib.ref_graph_export(h, off.ctypes.data, nb.ctypes.data, None)
    return off, nb[:n]


def test_update_host_graph_pins_batch_application():
    """The oracle's batch application (set semantics, updates in stream order)
    against the reference's updateHostGraph (cpuGraph.cpp:521-607), run on
    the same data graph batch after batch.  The reference applies a batch
    sorted by (src, dst) rather than in stream order, so the two agree on
    every batch that names each edge once: the generated batches, each edge
    kept at its first occurrence, are checked here; a batch that inserts and
    deletes one edge is order-dependent in the reference (recorded below)."""
    import dsm_b200 as d
    lib = _ref_graph_lib()
    w = d.Workload(2, scale_log2=-8, num_batches=6)
    q = w.queries[0]
    h = lib.ref_graph_new(w.nv, w.labels, len(w.edges), np.ascontiguousarray(w.edges.reshape(-1)))
    st = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
    try:
        for k, b in enumerate(w.batches()):
            keys = np.minimum(b[:, 1], b[:, 2]).astype(np.uint64) << 32 | np.maximum(b[:, 1], b[:, 2])
            _, first = np.unique(keys, return_index=True)
            b = np.ascontiguousarray(b[np.sort(first)])
            assert len(b) > 3000
            lib.ref_graph_update(h, len(b), np.ascontiguousarray(b.reshape(-1)))
            st.apply_graph(b)
            roff, rnb = _ref_export(lib, h, w.nv)
            ooff, onb = st.export()
            assert np.array_equal(roff, ooff) and np.array_equal(rnb, onb), f"batch {k}"
        # the recorded difference: insert then delete of one absent edge in
        # one batch -- in stream order the edge ends absent; the reference
        # sorts the two changes by (src, dst) only, so its outcome depends on
        # the sort's order of equal keys
        a, b_ = 0, 1
        while st.export()[1][st.export()[0][a]:st.export()[0][a + 1]].tolist().count(b_):
            b_ += 1
        pair = np.array([[1, a, b_, w.labels[a]], [0, a, b_, w.labels[a]]], np.uint32)
        st.apply_graph(pair)
        lib.ref_graph_update(h, 2, np.ascontiguousarray(pair.reshape(-1)))
        roff, rnb = _ref_export(lib, h, w.nv)
        ooff, onb = st.export()
        ref_has = b_ in rnb[roff[a]:roff[a + 1]].tolist()
        assert b_ not in onb[ooff[a]:ooff[a + 1]].tolist()
        print(f"insert+delete of one edge in a batch: reference keeps the edge: {ref_has}")
    finally:
        lib.ref_graph_free(h)


@pytest.mark.parametrize("ascending", [True, False])
def test_cluster_plan_against_reference(ascending):
    """The oracle's cluster-filter plan against the reference's own code:
    decycle, then getVertexCover / clustering (filter.cu:23-392) with
    encodingMeta::init (structure.cu:113-135) -- the clusters in order with
    their query vertices and validity, every merge and combine, the layer
    offsets -- and the position pick of clusterFilter (filter.cu:1582-1609),
    on the fixture's query shape and 60 random queries."""
    lib = C.CDLL(LIB)
    u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
    lib.ref_cluster_plan.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, C.c_uint32]
    merges = combines = 0
    for nq, edges in _queries(ascending):
        flat = np.array(edges, np.uint32).reshape(-1)
        out = np.zeros(1 << 16, np.uint32)
        n = lib.ref_cluster_plan(nq, len(edges), flat, out, len(out))
        assert n > 0
        qoff, qnbr = _csr_file_order(nq, edges)
        ours = orc.cluster_plan(qoff, qnbr)
        assert np.array_equal(ours, out[:n]), (nq, edges)
        merges += int(out[2])
        combines += int(out[3])
    assert merges > 50 and combines > 10  # the plans exercise merges and combines


def test_text_parsers_against_reference(tmp_path):
    """The engine's text reader and the oracle's parser against the
    reference's readGraphToCPUDynamic (io.cu:122-252) on generated files: the
    CSR in file order, the labels, and every batch's updates."""
    import dsm_b200 as d
    lib = C.CDLL(LIB)
    lib.ref_file_read.restype = C.c_void_p
    lib.ref_file_read.argtypes = [C.c_char_p, C.c_int]
    lib.ref_file_sizes.argtypes = [C.c_void_p] + [C.POINTER(C.c_uint32)] * 4
    lib.ref_file_export.argtypes = [C.c_void_p] + [C.c_void_p] * 5
    lib.ref_file_free.argtypes = [C.c_void_p]

    def ref_parse(path, isq):
        h = lib.ref_file_read(path.encode(), int(isq))
        try:
            nv, ne, nb, nu = (C.c_uint32() for _ in range(4))
            lib.ref_file_sizes(h, C.byref(nv), C.byref(ne), C.byref(nb), C.byref(nu))
            off = np.zeros(nv.value + 1, np.uint32)
            nbr = np.zeros(max(2 * ne.value, 1), np.uint32)
            lab = np.zeros(nv.value, np.uint32)
            sizes = np.zeros(max(nb.value, 1), np.uint32)
            ups = np.zeros(max(4 * nu.value, 1), np.uint32)
            lib.ref_file_export(h, off.ctypes.data, nbr.ctypes.data, lab.ctypes.data, sizes.ctypes.data,
                                ups.ctypes.data)
            return dict(offsets=off, nbrs=nbr[:2 * ne.value], labels=lab, batch_sizes=sizes[:nb.value],
                        updates=ups[:4 * nu.value].reshape(-1, 4))
        finally:
            lib.ref_file_free(h)

    for cfg, scale in ((1, 0), (2, -8)):
        w = d.Workload(cfg, scale_log2=scale, num_batches=4)
        w.write(str(tmp_path / f"q{cfg}_"), str(tmp_path / f"g{cfg}.in"))
        files = [(str(tmp_path / f"g{cfg}.in"), False)]
        files += [(str(tmp_path / f"q{cfg}_{k}.in"), True) for k in range(len(w.queries))]
        files += [(os.path.join(ROOT, "tests", "golden", n), n.startswith("example_q")) for n in
                  ("example_q_01.in", "example_g_01.in")]
        for path, isq in files:
            assert os.path.exists(path)  # the reference's reader exits the process on a missing file
            r = ref_parse(path, isq)
            a = d.TextGraph(path, isq)
            o = orc.parse(path, isq)
            for k in ("offsets", "nbrs", "labels", "batch_sizes", "updates"):
                assert np.array_equal(getattr(a, k), r[k]), (path, k)
                assert np.array_equal(o[k], r[k]), (path, k)
            if not isq:
                assert len(r["updates"]) > 0
