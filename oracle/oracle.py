"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker -- never by the engine.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB_PATH):
    build()
lib = C.CDLL(LIB_PATH)
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
P = C.c_void_p


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)


_sig("orc_file_parse", C.c_int, C.c_char_p, C.c_int, C.POINTER(P))
_sig("orc_file_free", None, P)
for n in ("nv", "ne", "num_batches", "num_updates"):
    _sig(f"orc_file_{n}", C.c_uint32, P)
for n in ("labels", "offsets", "nbrs", "edges", "batch_sizes", "updates"):
    _sig(f"orc_file_{n}", C.POINTER(C.c_uint32), P)
_sig("orc_decycle", C.c_int, C.c_uint32, u32p, u32p, u32p, u32p, u32p)
_sig("orc_order", C.c_int, C.c_uint32, u32p, u32p, C.c_uint32, C.c_uint32, u32p, u32p)
_sig("orc_cluster_plan", C.c_int, C.c_uint32, u32p, u32p, u32p, C.c_uint32)
_sig("orc_cluster_filter", C.c_int, C.c_uint32, u32p, u32p, u32p, C.c_uint32, u32p, u32p, u32p, P, P, P, P, P)
_sig("orc_stream_new", C.c_int, C.c_uint32, u32p, C.c_uint64, u32p, C.c_uint32, u32p, u32p, u32p, C.POINTER(P))
_sig("orc_stream_free", None, P)
_sig("orc_stream_apply", C.c_int, P, C.c_uint32, u32p, C.c_int)
_sig("orc_stream_apply_mt", C.c_int, P, C.c_uint32, u32p, C.c_int, C.c_int)
_sig("orc_stream_apply_graph", C.c_int, P, C.c_uint32, u32p)
_sig("orc_stream_set_query", C.c_int, P, C.c_uint32, u32p, u32p, u32p)
_sig("orc_stream_set_work_limit", None, P, C.c_uint64)
_sig("orc_stream_probe", C.c_uint64, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int)
_sig("orc_stream_set_budget", None, P, C.c_uint64)
_sig("orc_stream_complete", C.c_uint32, P)
_sig("orc_stream_sign", C.c_int8, P, C.c_uint32)
_sig("orc_stream_count", C.c_uint64, P, C.c_uint32)
_sig("orc_stream_tuples", C.POINTER(C.c_uint32), P, C.POINTER(C.c_uint64))
_sig("orc_stream_count_all", C.c_uint64, P)
_sig("orc_stream_export", C.c_uint64, P, P, P)
_sig("orc_stream_bytes", C.c_uint64, P)
_sig("orc_workload_generate", C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_uint32, C.POINTER(P))
_sig("orc_workload_free", None, P)
for n in ("nv", "num_queries", "num_batches", "num_updates"):
    _sig(f"orc_workload_{n}", C.c_uint32, P)
_sig("orc_workload_num_edges", C.c_uint64, P)
for n in ("labels", "edges", "batch_sizes", "updates"):
    _sig(f"orc_workload_{n}", C.POINTER(C.c_uint32), P)
_sig("orc_workload_query_nv", C.c_uint32, P, C.c_uint32)
for n in ("labels", "offsets", "nbrs"):
    _sig(f"orc_workload_query_{n}", C.POINTER(C.c_uint32), P, C.c_uint32)
_sig("orc_bruteforce_count", C.c_uint64, C.c_uint32, u32p, u32p, u32p, C.c_uint32, u32p, u32p, u32p)


def _u32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32))


def _arr(ptr, n):
    if n == 0:
        return np.zeros(0, np.uint32)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(np.uint32, copy=True)


def parse(path, is_query):
    h = P()
    if lib.orc_file_parse(path.encode(), int(is_query), C.byref(h)):
        raise ValueError(f"oracle: cannot parse {path}")
    try:
        nv, ne = lib.orc_file_nv(h), lib.orc_file_ne(h)
        out = dict(nv=nv, ne=ne, labels=_arr(lib.orc_file_labels(h), nv),
                   offsets=_arr(lib.orc_file_offsets(h), nv + 1), nbrs=_arr(lib.orc_file_nbrs(h), 2 * ne),
                   edges=_arr(lib.orc_file_edges(h), 2 * ne).reshape(-1, 2),
                   batch_sizes=_arr(lib.orc_file_batch_sizes(h), lib.orc_file_num_batches(h)),
                   updates=_arr(lib.orc_file_updates(h), 4 * lib.orc_file_num_updates(h)).reshape(-1, 4))
    finally:
        lib.orc_file_free(h)
    return out


def decycle(qoff, qnbr):
    qoff, qnbr = _u32(qoff), _u32(qnbr)
    nq = len(qoff) - 1
    toff = np.zeros(nq + 1, np.uint32)
    tnbr = np.zeros(max(len(qnbr), 1), np.uint32)
    tdeg = np.zeros(nq, np.uint32)
    n = lib.orc_decycle(nq, qoff, qnbr, toff, tnbr, tdeg)
    return toff, tnbr[:2 * n], tdeg


def order(qoff, qnbr, u, v):
    qoff, qnbr = _u32(qoff), _u32(qnbr)
    nq = len(qoff) - 1
    o = np.zeros(nq, np.uint32)
    b = np.zeros(nq, np.uint32)
    if lib.orc_order(nq, qoff, qnbr, u, v, o, b):
        raise ValueError("disconnected query")
    return o, b


def cluster_plan(qoff, qnbr):
    """The cluster plan of the decycled query, serialised (see oracle.h)."""
    nq = len(qoff) - 1
    out = np.zeros(1 << 16, np.uint32)
    n = lib.orc_cluster_plan(nq, _u32(qoff), _u32(qnbr), out, len(out))
    if n < 0:
        raise ValueError(f"cluster plan failed ({n})")
    return out[:n].copy()


def cluster_filter(qlabels, qoff, qnbr, nv, labels, off, nbr):
    """Candidate bitmaps (nq x ceil(nv/32)), v_cand_us, enc_pos_of_u, op plan."""
    qlabels, qoff, qnbr = _u32(qlabels), _u32(qoff), _u32(qnbr)
    labels, off, nbr = _u32(labels), _u32(off), _u32(nbr)
    if len(nbr) == 0:
        nbr = np.zeros(1, np.uint32)
    nq = len(qlabels)
    col = (nv + 31) // 32
    bm = np.zeros(nq * col, np.uint32)
    vc = np.zeros(nv, np.uint32)
    pos = np.zeros(nq, np.uint32)
    plan = np.zeros(4096, np.uint32)
    plen = C.c_uint32()
    rc = lib.orc_cluster_filter(nq, qlabels, qoff, qnbr, nv, labels, off, nbr, bm.ctypes.data, vc.ctypes.data,
                                pos.ctypes.data, plan.ctypes.data, C.byref(plen))
    if rc:
        raise ValueError(f"oracle filter: {rc}")
    return bm.reshape(nq, col), vc, pos, plan[:8 * plen.value].reshape(-1, 8)


class Stream:
    """Sequential per-update matcher over a data graph."""

    def __init__(self, nv, labels, edges, qlabels, qoff, qnbr):
        edges = _u32(edges).reshape(-1)
        if len(edges) == 0:
            edges = np.zeros(2, np.uint32)
            ne = 0
        else:
            ne = len(edges) // 2
        self.nq = len(qlabels)
        self.nv = nv
        h = P()
        rc = lib.orc_stream_new(nv, _u32(labels), ne, edges, self.nq, _u32(qlabels), _u32(qoff), _u32(qnbr),
                                C.byref(h))
        if rc:
            raise ValueError(f"oracle stream: {rc}")
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib.orc_stream_free(self._h)
            self._h = None

    def apply(self, updates, listed=True, threads=0):
        """Returns (signs[n], counts[n], list of (count, nq) arrays or None).
        threads > 0: the multi-threaded matcher on that many host threads
        (threads < 0: all cores); no work budget."""
        u = _u32(updates).reshape(-1)
        n = len(u) // 4
        if n == 0:
            return np.zeros(0, np.int8), np.zeros(0, np.uint64), []
        if threads:
            rc = lib.orc_stream_apply_mt(self._h, n, u, int(listed), max(threads, 0))
        else:
            rc = lib.orc_stream_apply(self._h, n, u, int(listed))
        if rc not in (0, 1):
            raise ValueError("oracle apply failed")
        # with a work budget, only the first `complete` updates have results
        self.complete = lib.orc_stream_complete(self._h)
        signs = np.array([lib.orc_stream_sign(self._h, i) for i in range(n)], np.int8)
        counts = np.array([lib.orc_stream_count(self._h, i) for i in range(n)], np.uint64)
        if not listed:
            return signs, counts, None
        tot = C.c_uint64()
        ptr = lib.orc_stream_tuples(self._h, C.byref(tot))
        flat = _arr(ptr, tot.value * self.nq).reshape(-1, self.nq)
        out, pos = [], 0
        for c in counts:
            k = 0 if int(c) >> 63 else int(c)  # a search over the work limit lists nothing
            out.append(flat[pos:pos + k])
            pos += k
        return signs, counts, out

    def apply_graph(self, updates):
        """Applies the updates to the graph without matching."""
        u = _u32(updates).reshape(-1)
        if len(u) and lib.orc_stream_apply_graph(self._h, len(u) // 4, u):
            raise ValueError("oracle apply failed")

    def set_query(self, qlabels, qoff, qnbr):
        """Replaces the query; the graph stays."""
        if lib.orc_stream_set_query(self._h, len(qlabels), _u32(qlabels), _u32(qoff), _u32(qnbr)):
            raise ValueError("oracle: bad query")
        self.nq = len(qlabels)

    def probe(self, op, a, b, threads=-1):
        """Count update (op, a, b) would report now; the graph is unchanged."""
        return lib.orc_stream_probe(self._h, int(op), int(a), int(b), int(threads))

    def set_work_limit(self, limit):
        """Per-update search bound (the engine's DSM_OPT_WORK_LIMIT)."""
        lib.orc_stream_set_work_limit(self._h, int(limit))

    def set_budget(self, nbytes):
        """Work budget (algorithmic bytes) of each later apply call."""
        lib.orc_stream_set_budget(self._h, int(nbytes))

    def count_all(self):
        return lib.orc_stream_count_all(self._h)

    def bytes(self):
        return lib.orc_stream_bytes(self._h)

    def export(self):
        off = np.zeros(self.nv + 1, np.uint32)
        n = lib.orc_stream_export(self._h, off.ctypes.data, None)
        nb = np.zeros(max(n, 1), np.uint32)
        lib.orc_stream_export(self._h, off.ctypes.data, nb.ctypes.data)
        return off, nb[:n]


def bruteforce_count(qlabels, qoff, qnbr, nv, labels, off, nbr):
    nbr = _u32(nbr)
    if len(nbr) == 0:
        nbr = np.zeros(1, np.uint32)
    return lib.orc_bruteforce_count(len(qlabels), _u32(qlabels), _u32(qoff), _u32(qnbr), nv, _u32(labels),
                                    _u32(off), nbr)


class Query:
    def __init__(self, labels, offsets, nbrs):
        self.labels, self.offsets, self.nbrs = _u32(labels), _u32(offsets), _u32(nbrs)

    @property
    def nv(self):
        return len(self.labels)


class Workload:
    """The engine's seeded workload (same generator source, compiled into the
    oracle library), for the CPU arms that must not load the engine."""

    def __init__(self, config, seed=0, scale_log2=0, num_batches=0):
        h = P()
        if lib.orc_workload_generate(config, seed, scale_log2, num_batches, C.byref(h)):
            raise ValueError("oracle: workload generation failed")
        try:
            self.nv = lib.orc_workload_nv(h)
            self.labels = _arr(lib.orc_workload_labels(h), self.nv)
            ne = lib.orc_workload_num_edges(h)
            self.edges = _arr(lib.orc_workload_edges(h), 2 * ne).reshape(-1, 2)
            self.queries = []
            for q in range(lib.orc_workload_num_queries(h)):
                nq = lib.orc_workload_query_nv(h, q)
                off = _arr(lib.orc_workload_query_offsets(h, q), nq + 1)
                self.queries.append(Query(_arr(lib.orc_workload_query_labels(h, q), nq), off,
                                          _arr(lib.orc_workload_query_nbrs(h, q), int(off[-1]))))
            self.batch_sizes = _arr(lib.orc_workload_batch_sizes(h), lib.orc_workload_num_batches(h))
            self.updates = _arr(lib.orc_workload_updates(h), 4 * lib.orc_workload_num_updates(h)).reshape(-1, 4)
        finally:
            lib.orc_workload_free(h)

    def batches(self):
        pos = 0
        for s in self.batch_sizes:
            yield self.updates[pos:pos + int(s)]
            pos += int(s)
