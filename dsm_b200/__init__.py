"""Python bindings of the B200 continuous subgraph matching engine.

Thin ctypes layer over ``include/dsm.h`` (the C ABI of ``libdsm.so``).  The
engine itself is C++/CUDA; this module only moves numpy arrays across the
boundary.  There is no CPU fallback: if the shared library is missing,
importing this package raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdsm.so")
CLI_PATH = os.path.join(HERE, "bin", "CDSM")

OK = 0
ERR = {1: "PARSE", 2: "OOM", 3: "OVERFLOW", 4: "TIMEOUT", 5: "LIMIT", 6: "ARG", 7: "CUDA", 8: "STATE",
       9: "NOT_FOUND"}

OPT_LIST, OPT_FILTER, OPT_RESULT_CAP, OPT_WARPS_PER_SM, OPT_DONATE, OPT_TIMEOUT_MS, OPT_LABEL_QUIRK, OPT_SORT, \
    OPT_LIST_LIMIT, OPT_MEM_BUDGET, OPT_SPLIT_MIN, OPT_DONATE_DEPTH, OPT_AUTOTUNE, OPT_GRAPH, OPT_STALL_TEST, \
    OPT_PLAIN, OPT_QUERY_LIST_LIMIT, OPT_WORK_LIMIT, OPT_PACK_MAX, OPT_FILTER_INCREMENTAL, OPT_MERGE_MAX, OPT_BFS_LEVELS, OPT_BFS_ROWS = range(1, 24)
INCOMPLETE = np.uint64(1 << 63)  # bit of a count whose search went over DSM_OPT_WORK_LIMIT

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run `python dsm_b200/build.py`")
lib = C.CDLL(LIB_PATH)

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
P = C.c_void_p


class Update(C.Structure):
    _fields_ = [("op", C.c_uint32), ("src", C.c_uint32), ("dst", C.c_uint32), ("label", C.c_uint32)]


class ResultView(C.Structure):
    _fields_ = [("batch_id", C.c_uint64), ("num_updates", C.c_uint32), ("num_queries", C.c_uint32),
                ("qids", C.POINTER(C.c_uint32)), ("widths", C.POINTER(C.c_uint32)),
                ("signs", C.POINTER(C.c_int8)), ("counts", C.POINTER(C.c_uint64)),
                ("offsets", C.POINTER(C.c_uint64)), ("tuples", C.POINTER(C.c_uint32)), ("listed", C.c_int),
                ("query_listed", C.POINTER(C.c_uint8))]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("batches", "updates", "matches", "seeds", "donations", "steals",
                                          "relocations", "result_regrows", "alg_bytes")] + \
               [(n, C.c_double) for n in ("last_batch_ms", "last_match_ms", "last_filter_ms", "last_update_ms",
                                          "last_sort_ms")] + [(n, C.c_uint64) for n in (
                   "device_bytes_in_use", "kernel_launches", "query_bytes", "live_queries", "tune_runs")] + \
               [("tune_best_ms", C.c_double)] + [(n, C.c_uint64) for n in (
                   "graph_launches", "graph_instantiations", "graph_captures", "compactions", "over_limit")]


class BatchTiming(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("queue_ms", "service_ms", "total_ms", "device_ms")] + \
               [(n, C.c_uint32) for n in ("merged_requests", "merged_updates")]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("dsm_status_string", C.c_char_p, C.c_int)
_sig("dsm_engine_create", C.c_int, C.c_int, C.c_size_t, C.POINTER(P))
_sig("dsm_engine_destroy", C.c_int, P)
_sig("dsm_last_error", C.c_char_p, P)
_sig("dsm_engine_set_option", C.c_int, P, C.c_int, C.c_int64)
_sig("dsm_engine_get_option", C.c_int, P, C.c_int, C.POINTER(C.c_int64))
_sig("dsm_graph_load", C.c_int, P, u32p, u32p, u32p, C.c_uint32)
_sig("dsm_graph_load_edges", C.c_int, P, C.c_uint32, u32p, C.c_uint64, u32p)
_sig("dsm_graph_export", C.c_int, P, P, P, C.POINTER(C.c_uint64))
_sig("dsm_graph_info", C.c_int, P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))
_sig("dsm_graph_apply", C.c_int, P, P, C.c_uint32)
_sig("dsm_query_register", C.c_int, P, u32p, u32p, u32p, C.c_uint32, C.POINTER(C.c_uint32))
_sig("dsm_query_retire", C.c_int, P, C.c_uint32)
_sig("dsm_query_live", C.c_int, P, P, C.c_uint32, C.POINTER(C.c_uint32))
_sig("dsm_query_order", C.c_int, P, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p)
_sig("dsm_query_filter", C.c_int, P, C.c_uint32, P, P)
_sig("dsm_query_filter_state", C.c_int, P, C.c_uint32, P, P, P)
_sig("dsm_query_plan", C.c_int, u32p, u32p, u32p, C.c_uint32, P, P, P, P, P)
_sig("dsm_batch_submit", C.c_int, P, P, C.c_uint32, C.POINTER(C.c_uint64))
_sig("dsm_batch_wait", C.c_int, P, C.c_uint64)
_sig("dsm_batch_results", C.c_int, P, C.c_uint64, C.POINTER(ResultView))
_sig("dsm_batch_release", C.c_int, P, C.c_uint64)
_sig("dsm_engine_stats", C.c_int, P, C.POINTER(Stats))
_sig("dsm_batch_timing_get", C.c_int, P, C.c_uint64, C.POINTER(BatchTiming))
_sig("dsm_serve_start", C.c_int, P, C.c_uint32)
_sig("dsm_engine_snapshot", C.c_int, P, C.c_char_p)
_sig("dsm_engine_resume", C.c_int, P, C.c_char_p)
_sig("dsm_serve_stop", C.c_int, P)
_sig("dsm_query_register_async", C.c_int, P, u32p, u32p, u32p, C.c_uint32, C.POINTER(C.c_uint64))
_sig("dsm_query_retire_async", C.c_int, P, C.c_uint32, C.POINTER(C.c_uint64))
_sig("dsm_query_admission", C.c_int, P, C.c_uint64, C.c_int64, C.POINTER(C.c_uint32))
_sig("dsm_text_read", C.c_int, C.c_char_p, C.c_int, C.POINTER(P), C.c_char_p, C.c_size_t)
_sig("dsm_text_free", None, P)
for _n in ("nv", "ne", "num_batches", "num_updates"):
    _sig(f"dsm_text_{_n}", C.c_uint32, P)
for _n in ("labels", "offsets", "nbrs", "edges", "batch_sizes"):
    _sig(f"dsm_text_{_n}", C.POINTER(C.c_uint32), P)
_sig("dsm_text_updates", C.POINTER(C.c_uint32), P)
_sig("dsm_text_write_binary", C.c_int, P, C.c_char_p)
_sig("dsm_workload_generate", C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_uint32, C.POINTER(P))
_sig("dsm_workload_free", None, P)
_sig("dsm_workload_nv", C.c_uint32, P)
_sig("dsm_workload_labels", C.POINTER(C.c_uint32), P)
_sig("dsm_workload_num_edges", C.c_uint64, P)
_sig("dsm_workload_edges", C.POINTER(C.c_uint32), P)
_sig("dsm_workload_num_queries", C.c_uint32, P)
_sig("dsm_workload_query_nv", C.c_uint32, P, C.c_uint32)
for _n in ("labels", "offsets", "nbrs"):
    _sig(f"dsm_workload_query_{_n}", C.POINTER(C.c_uint32), P, C.c_uint32)
_sig("dsm_workload_num_batches", C.c_uint32, P)
_sig("dsm_workload_batch_sizes", C.POINTER(C.c_uint32), P)
_sig("dsm_workload_num_updates", C.c_uint32, P)
_sig("dsm_workload_updates", C.POINTER(C.c_uint32), P)
_sig("dsm_workload_write", C.c_int, P, C.c_char_p, C.c_char_p)


class DSMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"DSM_ERR_{ERR.get(code, code)}: {msg}")
        self.code = code


def _arr(ptr, n, dtype=np.uint32):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _u32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint32))


class Query:
    """A query graph in the reference's CSR-in-file-order form."""

    def __init__(self, labels, offsets, nbrs):
        self.labels = _u32(labels)
        self.offsets = _u32(offsets)
        self.nbrs = _u32(nbrs)

    @property
    def nv(self):
        return len(self.labels)

    @classmethod
    def from_edges(cls, labels, edges):
        labels = _u32(labels)
        nq = len(labels)
        deg = np.zeros(nq, np.int64)
        for a, b in edges:
            deg[a] += 1
            deg[b] += 1
        off = np.zeros(nq + 1, np.uint32)
        off[1:] = np.cumsum(deg)
        fill = off[:-1].astype(np.int64).copy()
        nb = np.zeros(off[-1], np.uint32)
        for a, b in edges:
            nb[fill[a]] = b
            fill[a] += 1
            nb[fill[b]] = a
            fill[b] += 1
        return cls(labels, off, nb)


class TextGraph:
    """A query or data file in the reference's text format (io.cu:122-252)."""

    def __init__(self, path, is_query):
        h = P()
        err = C.create_string_buffer(512)
        rc = lib.dsm_text_read(path.encode(), int(is_query), C.byref(h), err, 512)
        if rc:
            raise DSMError(rc, err.value.decode())
        try:
            self.nv = lib.dsm_text_nv(h)
            self.ne = lib.dsm_text_ne(h)
            self.labels = _arr(lib.dsm_text_labels(h), self.nv)
            self.offsets = _arr(lib.dsm_text_offsets(h), self.nv + 1)
            self.nbrs = _arr(lib.dsm_text_nbrs(h), 2 * self.ne)
            self.edges = _arr(lib.dsm_text_edges(h), 2 * self.ne).reshape(-1, 2)
            nb = lib.dsm_text_num_batches(h)
            self.batch_sizes = _arr(lib.dsm_text_batch_sizes(h), nb)
            nu = lib.dsm_text_num_updates(h)
            self.updates = _arr(lib.dsm_text_updates(h), 4 * nu).reshape(-1, 4)
        finally:
            lib.dsm_text_free(h)

    def query(self):
        return Query(self.labels, self.offsets, self.nbrs)


def to_binary(path, out_path, is_query):
    """Converts a query or data file (text or binary) to the binary form,
    which the engine and CDSM then map instead of parsing."""
    h = P()
    err = C.create_string_buffer(512)
    rc = lib.dsm_text_read(path.encode(), int(is_query), C.byref(h), err, 512)
    if rc:
        raise DSMError(rc, err.value.decode())
    try:
        rc = lib.dsm_text_write_binary(h, out_path.encode())
        if rc:
            raise DSMError(rc, f"cannot write {out_path}")
    finally:
        lib.dsm_text_free(h)


class Workload:
    """Seeded synthetic workload (configs 1-5)."""

    def __init__(self, config, seed=0, scale_log2=0, num_batches=0):
        h = P()
        rc = lib.dsm_workload_generate(config, seed, scale_log2, num_batches, C.byref(h))
        if rc:
            raise DSMError(rc, "workload generation failed")
        self._h = h
        self.nv = lib.dsm_workload_nv(h)
        self.labels = _arr(lib.dsm_workload_labels(h), self.nv)
        ne = lib.dsm_workload_num_edges(h)
        self.edges = _arr(lib.dsm_workload_edges(h), 2 * ne).reshape(-1, 2)
        self.queries = []
        for q in range(lib.dsm_workload_num_queries(h)):
            nq = lib.dsm_workload_query_nv(h, q)
            off = _arr(lib.dsm_workload_query_offsets(h, q), nq + 1)
            self.queries.append(Query(_arr(lib.dsm_workload_query_labels(h, q), nq), off,
                                      _arr(lib.dsm_workload_query_nbrs(h, q), int(off[-1]))))
        nb = lib.dsm_workload_num_batches(h)
        self.batch_sizes = _arr(lib.dsm_workload_batch_sizes(h), nb)
        nu = lib.dsm_workload_num_updates(h)
        self.updates = _arr(lib.dsm_workload_updates(h), 4 * nu).reshape(-1, 4)

    def batches(self):
        pos = 0
        for s in self.batch_sizes:
            yield self.updates[pos:pos + int(s)]
            pos += int(s)

    def write(self, query_prefix, data_path):
        rc = lib.dsm_workload_write(self._h, query_prefix.encode(), data_path.encode())
        if rc:
            raise DSMError(rc, "write failed")

    def __del__(self):
        if getattr(self, "_h", None):
            lib.dsm_workload_free(self._h)
            self._h = None


def query_plan(q):
    """Host-side plan of a query (no GPU): orders per ordered query edge."""
    nq = q.nv
    ne2 = int(q.offsets[-1])
    orders = np.zeros(ne2 * nq, np.uint32)
    bn = np.zeros(ne2 * nq, np.uint32)
    n_oe = C.c_uint32()
    pos = np.zeros(nq, np.uint32)
    oedges = np.zeros(2 * ne2, np.uint32)
    rc = lib.dsm_query_plan(q.offsets, q.nbrs, q.labels, nq, orders.ctypes.data, bn.ctypes.data,
                            oedges.ctypes.data, C.byref(n_oe), pos.ctypes.data)
    if rc:
        raise DSMError(rc, "query plan failed")
    k = n_oe.value
    return {"orders": orders[:k * nq].reshape(k, nq), "bn": bn[:k * nq].reshape(k, nq),
            "oedges": oedges[:2 * k].reshape(k, 2), "enc_pos_of_u": pos}


class BatchResult:
    """Per (query, update) canonically sorted tuples of one batch."""

    def __init__(self, view):
        n, nq = view.num_updates, view.num_queries
        self.batch_id = view.batch_id
        self.qids = _arr(view.qids, nq)
        self.widths = _arr(view.widths, nq)
        self.signs = _arr(view.signs, n, np.int8)
        self.counts = _arr(view.counts, nq * n, np.uint64).reshape(nq, n) if nq else np.zeros((0, n), np.uint64)
        self.offsets = _arr(view.offsets, nq * n + 1, np.uint64)
        self.tuples = _arr(view.tuples, int(self.offsets[-1]) if len(self.offsets) else 0)
        self.listed = bool(view.listed)
        self.query_listed = _arr(view.query_listed, nq, np.uint8).astype(bool)
        self.num_updates = n

    @property
    def complete(self):
        """(queries, updates) mask: the count is exact (not over the work limit)."""
        return (self.counts & INCOMPLETE) == 0

    def exact_matches(self):
        return int(self.counts[self.complete].sum())

    def query_index(self, qid):
        return int(np.nonzero(self.qids == qid)[0][0])

    def tuples_of(self, qid, i):
        """(count, width) array of update i's embeddings for query qid."""
        ql = self.query_index(qid)
        s = ql * self.num_updates + i
        w = int(self.widths[ql])
        return self.tuples[int(self.offsets[s]):int(self.offsets[s + 1])].reshape(-1, w)


class Engine:
    def __init__(self, device=0, mem_budget=0):
        h = P()
        rc = lib.dsm_engine_create(device, mem_budget, C.byref(h))
        if rc:
            raise DSMError(rc, "engine create failed")
        self._h = h

    def _ck(self, rc):
        if rc:
            raise DSMError(rc, lib.dsm_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib.dsm_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_option(self, opt, value):
        self._ck(lib.dsm_engine_set_option(self._h, opt, int(value)))

    def get_option(self, opt):
        v = C.c_int64()
        self._ck(lib.dsm_engine_get_option(self._h, opt, C.byref(v)))
        return v.value

    def load_graph_edges(self, nv, labels, edges):
        edges = _u32(edges).reshape(-1)
        self._ck(lib.dsm_graph_load_edges(self._h, nv, _u32(labels), len(edges) // 2, edges))

    def load_graph_csr(self, offsets, nbrs, labels):
        self._ck(lib.dsm_graph_load(self._h, _u32(offsets), _u32(nbrs), _u32(labels), len(labels)))

    def apply_graph(self, updates):
        """Applies updates to the device graph without matching."""
        u = self.pack_updates(updates)
        self._ck(lib.dsm_graph_apply(self._h, u.ctypes.data, len(u)))

    def graph_info(self):
        nv, ne, aw = C.c_uint32(), C.c_uint64(), C.c_uint64()
        self._ck(lib.dsm_graph_info(self._h, C.byref(nv), C.byref(ne), C.byref(aw)))
        return {"nv": nv.value, "num_entries": ne.value, "arena_words": aw.value}

    def export_graph(self):
        n = C.c_uint64()
        nv = C.c_uint32()
        self._ck(lib.dsm_graph_info(self._h, C.byref(nv), None, None))
        off = np.zeros(nv.value + 1, np.uint32)
        self._ck(lib.dsm_graph_export(self._h, off.ctypes.data, None, C.byref(n)))
        nb = np.zeros(max(n.value, 1), np.uint32)
        self._ck(lib.dsm_graph_export(self._h, off.ctypes.data, nb.ctypes.data, C.byref(n)))
        return off, nb[:n.value]

    def register(self, q):
        qid = C.c_uint32()
        self._ck(lib.dsm_query_register(self._h, q.offsets, q.nbrs, q.labels, q.nv, C.byref(qid)))
        return qid.value

    def retire(self, qid):
        self._ck(lib.dsm_query_retire(self._h, qid))

    def live_queries(self):
        n = C.c_uint32()
        self._ck(lib.dsm_query_live(self._h, None, 0, C.byref(n)))
        ids = np.zeros(max(n.value, 1), np.uint32)
        self._ck(lib.dsm_query_live(self._h, ids.ctypes.data, len(ids), C.byref(n)))
        return ids[:n.value].tolist()

    def order(self, qid, u, v, nq):
        o = np.zeros(nq, np.uint32)
        b = np.zeros(nq, np.uint32)
        self._ck(lib.dsm_query_order(self._h, qid, u, v, o, b))
        return o, b

    def filter(self, qid, nq, nv):
        col = (nv + 31) // 32
        bm = np.zeros(nq * col, np.uint32)
        vc = np.zeros(nv, np.uint32)
        self._ck(lib.dsm_query_filter(self._h, qid, bm.ctypes.data, vc.ctypes.data))
        return bm.reshape(nq, col), vc

    def filter_state(self, qid, nq, nv):
        """The resident filter state of query qid after the last batch:
        bitmaps, LDF+NLF masks, and (full recompute?, vertices recomputed)."""
        col = (nv + 31) // 32
        bm = np.zeros(nq * col, np.uint32)
        vc = np.zeros(nv, np.uint32)
        info = np.zeros(2, np.uint32)
        self._ck(lib.dsm_query_filter_state(self._h, qid, bm.ctypes.data, vc.ctypes.data, info.ctypes.data))
        return bm.reshape(nq, col), vc, (bool(info[0]), int(info[1]))

    @staticmethod
    def pack_updates(updates):
        u = np.ascontiguousarray(np.asarray(updates, dtype=np.uint32).reshape(-1, 4))
        return u

    def submit(self, updates):
        u = self.pack_updates(updates)
        bid = C.c_uint64()
        self._ck(lib.dsm_batch_submit(self._h, u.ctypes.data, len(u), C.byref(bid)))
        return bid.value

    def results(self, bid, release=True):
        v = ResultView()
        self._ck(lib.dsm_batch_results(self._h, bid, C.byref(v)))
        r = BatchResult(v)
        if release:
            self._ck(lib.dsm_batch_release(self._h, bid))
        return r

    def run_batch(self, updates):
        return self.results(self.submit(updates))

    def wait(self, bid):
        self._ck(lib.dsm_batch_wait(self._h, bid))

    def timing(self, bid):
        t = BatchTiming()
        self._ck(lib.dsm_batch_timing_get(self._h, bid, C.byref(t)))
        return {f: getattr(t, f) for f, _ in BatchTiming._fields_}

    def snapshot(self, path):
        self._ck(lib.dsm_engine_snapshot(self._h, path.encode()))

    def resume(self, path):
        self._ck(lib.dsm_engine_resume(self._h, path.encode()))

    # serving loop
    def serve_start(self, max_merge_updates=0):
        self._ck(lib.dsm_serve_start(self._h, max_merge_updates))

    def serve_stop(self):
        self._ck(lib.dsm_serve_stop(self._h))

    def register_async(self, q):
        t = C.c_uint64()
        self._ck(lib.dsm_query_register_async(self._h, q.offsets, q.nbrs, q.labels, q.nv, C.byref(t)))
        return t.value

    def retire_async(self, qid):
        t = C.c_uint64()
        self._ck(lib.dsm_query_retire_async(self._h, qid, C.byref(t)))
        return t.value

    def admission(self, ticket, timeout_ms=-1):
        """qid once admitted; None while the registration still waits."""
        qid = C.c_uint32()
        rc = lib.dsm_query_admission(self._h, ticket, int(timeout_ms), C.byref(qid))
        if rc == 4:  # DSM_ERR_TIMEOUT
            return None
        self._ck(rc)
        return qid.value

    def stats(self):
        s = Stats()
        self._ck(lib.dsm_engine_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in Stats._fields_}
