"""Shared test helpers: run the engine and the oracle side by side."""
import numpy as np

from oracle import oracle as orc


def oracle_stream(nv, labels, edges, q):
    return orc.Stream(nv, labels, edges, q.labels, q.offsets, q.nbrs)


def compare_batch(res, qid, signs, counts, tuples, tag=""):
    """Engine batch result for query qid == oracle output, update by update."""
    n = len(signs)
    assert res.num_updates == n, tag
    assert np.array_equal(res.signs, signs), f"{tag}: signs differ"
    ql = res.query_index(qid)
    got_counts = res.counts[ql]
    bad = np.nonzero(got_counts != counts)[0]
    assert len(bad) == 0, f"{tag}: counts differ at updates {bad[:10]}: engine {got_counts[bad[:10]]} oracle {counts[bad[:10]]}"
    if tuples is not None and res.listed:
        for i in range(n):
            t = res.tuples_of(qid, i)
            assert np.array_equal(t, tuples[i]), f"{tag}: update {i} tuples differ\n{t[:5]}\n{tuples[i][:5]}"


def run_stream(eng, qids, streams, batches, check_graph_every=0, listed=True):
    """Submits each batch to the engine and the oracle streams; compares."""
    total = 0
    for b, ups in enumerate(batches):
        res = eng.run_batch(ups)
        for qid, st in zip(qids, streams):
            s, c, t = st.apply(ups, listed=listed)
            compare_batch(res, qid, s, c, t, tag=f"batch {b} query {qid}")
            total += int(c.sum())
        if check_graph_every and (b + 1) % check_graph_every == 0:
            off, nb = eng.export_graph()
            ooff, onb = streams[0].export()
            assert np.array_equal(off, ooff) and np.array_equal(nb, onb), f"graph differs after batch {b}"
    return total
