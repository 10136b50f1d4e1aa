"""Shared test helpers: run the engine and the oracle side by side.

The oracle enumerates ~15M embeddings/s on one core while some updates of
the config-2/3 workloads carry 10^8 or more, so the oracle runs with a work
budget per slice of updates: it applies every update to its graph, but
enumerates only while the slice's budget lasts (`Stream.complete` updates
have results).  The engine always runs whole batches; the comparison covers
every update the oracle could afford, and the graphs are compared in full."""
import functools

import numpy as np

from oracle import oracle as orc


@functools.lru_cache(maxsize=None)
def _generated(config, seed, scale_log2, num_batches):
    import dsm_b200 as d
    return d.Workload(config, seed=seed, scale_log2=scale_log2, num_batches=num_batches)


class _FirstBatches:
    """The first `nb` batches of a generated workload (the update stream is
    generated in order, so it equals a workload generated with nb batches)."""

    def __init__(self, w, nb):
        self._w = w
        self.nv, self.labels, self.edges, self.queries = w.nv, w.labels, w.edges, w.queries
        self.batch_sizes = w.batch_sizes[:nb]
        self.updates = w.updates[:int(self.batch_sizes.sum())]

    def batches(self):
        pos = 0
        for s in self.batch_sizes:
            yield self.updates[pos:pos + int(s)]
            pos += int(s)


def workload(config, seed=0, scale_log2=0, num_batches=0):
    """A seeded workload, generated once per test session (generation screens
    query candidates on the host and takes seconds to minutes; the tests only
    read it)."""
    if num_batches == 0:
        return _generated(config, seed, scale_log2, 0)
    return _FirstBatches(_generated(config, seed, scale_log2, max(num_batches, 3)), num_batches)


BYTES_PER_EMBEDDING = 64  # work budget per embedding the oracle is allowed


def oracle_stream(nv, labels, edges, q):
    return orc.Stream(nv, labels, edges, q.labels, q.offsets, q.nbrs)


def oracle_prefix(nv, labels, edges, q, ups, limit):
    """Updates of `ups` a fresh oracle enumerates within ~`limit` embeddings."""
    st = oracle_stream(nv, labels, edges, q)
    st.set_budget(BYTES_PER_EMBEDDING * limit)
    st.apply(ups, listed=False)
    return st.complete


def oracle_apply(st, ups, listed, limit=None, slice_len=64):
    """Applies a batch to the oracle in slices; returns signs, counts, tuples
    (list per update, or None) and the mask of updates with results."""
    n = len(ups)
    if limit is None:
        s, c, t = st.apply(ups, listed=listed)
        return s, c, t, np.ones(n, bool)
    st.set_budget(BYTES_PER_EMBEDDING * limit)
    signs, counts, tuples, valid = [], [], [], []
    for i in range(0, n, slice_len):
        sl = ups[i:i + slice_len]
        s, c, t = st.apply(sl, listed=listed)
        v = np.zeros(len(sl), bool)
        v[:st.complete] = True
        signs.append(s)
        counts.append(c)
        valid.append(v)
        if listed:
            tuples += t
    st.set_budget(2 ** 63)
    if n == 0:
        return np.zeros(0, np.int8), np.zeros(0, np.uint64), ([] if listed else None), np.zeros(0, bool)
    return (np.concatenate(signs), np.concatenate(counts), tuples if listed else None, np.concatenate(valid))


def compare_batch(res, qid, signs, counts, tuples, valid=None, tag=""):
    """Engine batch result for query qid == oracle output, update by update
    (only where `valid`)."""
    n = len(signs)
    if valid is None:
        valid = np.ones(n, bool)
    assert res.num_updates == n, tag
    assert np.array_equal(res.signs, signs), f"{tag}: signs differ"
    ql = res.query_index(qid)
    got = res.counts[ql]
    bad = np.nonzero((got != counts) & valid)[0]
    assert len(bad) == 0, f"{tag}: counts differ at updates {bad[:10]}: engine {got[bad[:10]]} oracle {counts[bad[:10]]}"
    if tuples is not None and res.listed:
        for i in np.nonzero(valid)[0]:
            t = res.tuples_of(qid, int(i))
            assert np.array_equal(t, tuples[i]), f"{tag}: update {i} tuples differ\n{t[:5]}\n{tuples[i][:5]}"
    return int(valid.sum())


def run_stream(eng, qids, streams, batches, check_graph_every=0, listed=True, limit=None):
    """Submits each batch to the engine and the oracle streams; compares.
    Returns (embeddings compared, updates compared)."""
    total, checked = 0, 0
    for b, ups in enumerate(batches):
        res = eng.run_batch(ups)
        for qid, st in zip(qids, streams):
            s, c, t, v = oracle_apply(st, ups, listed, limit)
            checked += compare_batch(res, qid, s, c, t, v, tag=f"batch {b} query {qid}")
            total += int(c[v].sum())
        if check_graph_every and (b + 1) % check_graph_every == 0:
            off, nb = eng.export_graph()
            ooff, onb = streams[0].export()
            assert np.array_equal(off, ooff) and np.array_equal(nb, onb), f"graph differs after batch {b}"
    return total, checked
