"""dsm_count_edge_embeddings_noalloc, the entry point for callers that cannot
allocate device memory (a framework that owns the device allocator, or a
thread that must not synchronise the device with cudaMalloc / cudaFree).

The graph, updates and output are device buffers owned by the test (torch
tensors, as such a caller's framework would own them); the entry point itself
allocates nothing.  Its counts must equal what the engine's regular path
reports for the same edges, on two calls in a row (the second call reuses the
static scratch the first one left behind).  This file is collected last."""
import ctypes as C
import time

import numpy as np
import pytest

import dsm_b200 as d

pytestmark = pytest.mark.gpu


def _device_graph(nv, edges):
    """The documented layout: per vertex {run start in 16-byte units, degree},
    runs sorted and padded to 4 entries."""
    adj_lists = [[] for _ in range(nv)]
    for a, b in edges:
        adj_lists[a].append(int(b))
        adj_lists[b].append(int(a))
    adj = np.zeros(2 * nv, np.uint32)
    runs, start16 = [], 0
    for v in range(nv):
        lst = sorted(set(adj_lists[v]))
        cap = (len(lst) + 3) // 4 * 4
        adj[2 * v], adj[2 * v + 1] = start16, len(lst)
        runs.append(np.array(lst + [0xFFFFFFFF] * (cap - len(lst)), np.uint32))
        start16 += cap // 4
    arena = np.concatenate(runs) if runs else np.zeros(4, np.uint32)
    return adj, arena


def _engine_counts(w, q, pick):
    """Counts from the regular engine path: each picked edge is deleted and
    re-inserted, so every delete sees the unchanged graph."""
    e = d.Engine(0)
    e.set_option(d.OPT_LIST, 0)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(q)
    ups = []
    for a, b in pick:
        ups.append([0, a, b, 0])
        ups.append([1, a, b, 0])
    r = e.run_batch(np.array(ups, np.uint32))
    counts = r.counts[r.query_index(qid)][0::2].astype(np.uint64)
    e.close()
    return counts


def _entry():
    f = d.lib.dsm_count_edge_embeddings_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    return f


def test_noalloc_counts_match_engine_twice():
    torch = pytest.importorskip("torch")
    f = _entry()

    w = d.Workload(1)
    q = w.queries[0]
    adj, arena = _device_graph(w.nv, w.edges)
    dev = torch.device("cuda", 0)
    t_adj = torch.from_numpy(adj.view(np.int32)).to(dev)
    t_arena = torch.from_numpy(arena.view(np.int32)).to(dev)
    t_lab = torch.from_numpy(w.labels.view(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(11)

    for call in range(2):
        pick = w.edges[rng.choice(len(w.edges), 300, replace=False)]
        ups = np.zeros((len(pick), 4), np.uint32)
        ups[:, 0] = 1
        ups[:, 1:3] = pick
        t_ups = torch.from_numpy(ups.view(np.int32).reshape(-1)).to(dev)
        t_cnt = torch.full((len(pick),), -1, dtype=torch.int64, device=dev)  # stale values must not leak
        torch.cuda.synchronize()
        rc = f(0, w.nv, t_adj.data_ptr(), t_arena.data_ptr(), t_lab.data_ptr(), q.offsets.ctypes.data,
               q.nbrs.ctypes.data, q.labels.ctypes.data, q.nv, t_ups.data_ptr(), len(pick), t_cnt.data_ptr(),
               C.c_void_p(stream))
        assert rc == 0, d.lib.dsm_status_string(rc)
        got = t_cnt.cpu().numpy().view(np.uint64)
        want = _engine_counts(w, q, pick)
        assert np.array_equal(got, want), f"call {call}: {np.nonzero(got != want)[0][:10]}"
        assert want.sum() > 0

    # sizes beyond the stated maximum are refused before anything runs
    big = torch.zeros(4 * 4097, dtype=torch.int32, device=dev)
    out = torch.zeros(4097, dtype=torch.int64, device=dev)
    rc = f(0, w.nv, t_adj.data_ptr(), t_arena.data_ptr(), t_lab.data_ptr(), q.offsets.ctypes.data,
           q.nbrs.ctypes.data, q.labels.ctypes.data, q.nv, big.data_ptr(), 4097, out.data_ptr(), C.c_void_p(stream))
    assert rc == 5  # DSM_ERR_LIMIT


def test_noalloc_edge_cases():
    """Empty call, a query whose labels meet no edge (no seeds: the matcher
    finishes at once), ids out of range and self loops (count 0, no graph
    read), and a query above the 8-vertex limit (refused)."""
    torch = pytest.importorskip("torch")
    f = _entry()
    w = d.Workload(1)
    q = w.queries[0]
    adj, arena = _device_graph(w.nv, w.edges)
    dev = torch.device("cuda", 0)
    t_adj = torch.from_numpy(adj.view(np.int32)).to(dev)
    t_arena = torch.from_numpy(arena.view(np.int32)).to(dev)
    t_lab = torch.from_numpy(w.labels.view(np.int32)).to(dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def call(qq, ups):
        ups = np.asarray(ups, np.uint32).reshape(-1, 4)
        t_ups = torch.from_numpy(ups.view(np.int32).reshape(-1).copy()).to(dev) if len(ups) else \
            torch.zeros(4, dtype=torch.int32, device=dev)
        out = torch.full((max(len(ups), 1),), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()
        rc = f(0, w.nv, t_adj.data_ptr(), t_arena.data_ptr(), t_lab.data_ptr(), qq.offsets.ctypes.data,
               qq.nbrs.ctypes.data, qq.labels.ctypes.data, qq.nv, t_ups.data_ptr(), len(ups), out.data_ptr(),
               stream)
        return rc, out.cpu().numpy().view(np.uint64)[:len(ups)]

    rc, _ = call(q, [])
    assert rc == 0
    # labels 0..3 only in the graph: a query of label 7 has no seed
    q7 = d.Query(np.full(q.nv, 7, np.uint32), q.offsets, q.nbrs)
    pick = w.edges[:64]
    ups = np.zeros((64, 4), np.uint32)
    ups[:, 0] = 1
    ups[:, 1:3] = pick
    t0 = time.perf_counter()
    rc, got = call(q7, ups)
    assert rc == 0 and not got.any()
    assert time.perf_counter() - t0 < 2.0  # no bounded wait ran out
    # a live edge, then ids >= nv and a self loop: those count 0
    a, b = (int(x) for x in w.edges[0])
    bad = [[1, a, b, 0], [1, w.nv, b, 0], [1, a, w.nv + 5, 0], [1, 0xFFFFFFFF, 0xFFFFFFFF, 0], [1, a, a, 0]]
    rc, got = call(q, bad)
    assert rc == 0
    assert got[1:].tolist() == [0, 0, 0, 0]
    assert got[0] == _engine_counts(w, q, np.array([[a, b]], np.uint32))[0]
    # nine query vertices: beyond the stated maximum of eight
    q9 = d.Query.from_edges(np.zeros(9, np.uint32), [(i, i + 1) for i in range(8)])
    rc, _ = call(q9, ups[:4])
    assert rc == 5  # DSM_ERR_LIMIT
