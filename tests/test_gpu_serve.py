"""The serving loop (continuous batching, admission by memory budget).

Batches queued while the engine is busy run as one device batch; every
update's embeddings must still equal the oracle's sequential result.  A query
served in a mix with other queries (registered and retired while batches
flow) must get exactly the results it gets alone.  Admission charges each
query its device footprint: registrations beyond the budget wait until a
retirement or a larger budget makes room, first come first served."""
import numpy as np
import pytest

import dsm_b200 as d
from tests.helpers import compare_batch, oracle_apply, oracle_stream, workload

pytestmark = pytest.mark.gpu


def test_merged_batches_equal_oracle():
    w = workload(1)
    q = w.queries[0]
    e = d.Engine(0)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(q)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    e.serve_start()
    ups = w.updates
    chunks = [ups[i:i + 64] for i in range(0, len(ups), 64)]
    bids = [e.submit(c) for c in chunks]  # queued while the first ones run
    merged = 1
    for b, (bid, c) in enumerate(zip(bids, chunks)):
        t = e.timing(bid)
        merged = max(merged, t["merged_requests"])
        assert t["total_ms"] >= t["queue_ms"] >= 0 and t["merged_updates"] >= len(c)
        res = e.results(bid)
        s, cnt, tup, v = oracle_apply(st, c, True)
        compare_batch(res, qid, s, cnt, tup, v, tag=f"request {b}")
    e.serve_stop()
    assert merged > 1, "no two queued batches were served by one device batch"
    off, nb = e.export_graph()
    ooff, onb = st.export()
    assert np.array_equal(off, ooff) and np.array_equal(nb, onb)
    e.close()


def test_alone_equals_mix_with_churn():
    w = workload(3, scale_log2=-6, num_batches=2)
    ups = np.concatenate([b[:512] for b in w.batches()])
    chunks = [ups[i:i + 128] for i in range(0, len(ups), 128)]
    qs = w.queries[:16]
    target = qs[0]

    alone = d.Engine(0)
    alone.load_graph_edges(w.nv, w.labels, w.edges)
    aq = alone.register(target)
    ref = [alone.run_batch(c) for c in chunks]
    alone.close()

    mix = d.Engine(0)
    mix.load_graph_edges(w.nv, w.labels, w.edges)
    mix.serve_start()
    qids = [mix.register(q) for q in qs]  # through the queue
    mq = qids[0]
    bids = []
    old = new = None
    for k, c in enumerate(chunks):
        bids.append(mix.submit(c))
        if k == 1:
            old = qids[5]
            mix.retire(old)  # takes effect between device batches
        if k == 2:
            new = mix.register(w.queries[20])  # may reuse the retired id
    for k, (bid, r) in enumerate(zip(bids, ref)):
        res = mix.results(bid)
        live = res.qids.tolist()
        assert mq in live and len(live) == (16 if k != 2 else 15)
        if k <= 1:
            assert old in live
        elif k == 2:
            assert old not in live and new not in live
        else:
            assert new in live
        a, b = r.query_index(aq), res.query_index(mq)
        assert np.array_equal(res.signs, r.signs)
        assert np.array_equal(res.counts[b], r.counts[a]), f"request {k}: counts differ"
        for i in range(len(chunks[k])):
            assert np.array_equal(res.tuples_of(mq, i), r.tuples_of(aq, i)), f"request {k} update {i}"
    mix.serve_stop()
    mix.close()


def test_admission_waits_for_memory():
    w = workload(1)
    q = w.queries[0]
    e = d.Engine(0)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    warm = [e.register(q) for _ in range(3)]
    e.run_batch(w.updates[:32])  # batch scratch sized for three live queries
    for x in warm[1:]:
        e.retire(x)
    q1 = warm[0]
    s = e.stats()
    f, base = s["query_bytes"], s["device_bytes_in_use"]
    assert f > 0 and s["live_queries"] == 1
    e.set_option(d.OPT_MEM_BUDGET, base + int(2.5 * f))  # room for two queries
    e.serve_start()
    t2, t3, t4 = e.register_async(q), e.register_async(q), e.register_async(q)
    q2 = e.admission(t2, 10_000)
    assert q2 is not None
    assert e.admission(t3, 300) is None  # waits for memory
    e.retire(q1)  # frees one query's footprint: t3 gets it
    q3 = e.admission(t3, 10_000)
    assert q3 is not None
    assert e.admission(t4, 300) is None
    e.set_option(d.OPT_MEM_BUDGET, base + int(3.5 * f))  # a larger budget admits t4
    q4 = e.admission(t4, 10_000)
    assert q4 is not None
    res = e.results(e.submit(w.updates[32:64]))
    assert sorted(res.qids.tolist()) == sorted([q2, q3, q4])
    # a query that could never fit fails at once
    e.set_option(d.OPT_MEM_BUDGET, e.stats()["device_bytes_in_use"] + f // 2)
    t5 = e.register_async(q)
    with pytest.raises(d.DSMError) as ex:
        e.admission(t5, 10_000)
    assert ex.value.code == 2  # DSM_ERR_OOM
    e.serve_stop()
    e.close()


def test_serving_errors_and_restart():
    w = workload(1)
    e = d.Engine(0)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(w.queries[0])
    e.serve_start()
    with pytest.raises(d.DSMError):
        e.serve_start()
    with pytest.raises(d.DSMError):
        e.submit([[1, 0, w.nv, 0]])  # vertex out of range: refused at submit
    bid = e.submit(np.zeros((0, 4), np.uint32))
    assert e.results(bid).num_updates == 0
    e.serve_stop()
    e.serve_stop()
    r = e.run_batch(w.updates[:8])  # plain form again
    assert r.num_updates == 8 and qid in r.qids.tolist()
    e.close()


def test_snapshot_resume(tmp_path):
    """An engine resumed from a snapshot (graph, queries with their ids, batch
    counter) gives the same results for the rest of the stream as the engine
    that wrote it."""
    w = workload(1)
    ups = w.updates
    half = len(ups) // 2
    a = d.Engine(0)
    a.load_graph_edges(w.nv, w.labels, w.edges)
    tri = d.Query.from_edges([0, 1, 2], [(0, 1), (1, 2), (0, 2)])
    ids = [a.register(w.queries[0]), a.register(tri), a.register(tri)]
    a.retire(ids[1])  # a hole in the ids
    for i in range(0, half, 256):
        a.run_batch(ups[i:min(i + 256, half)])
    path = str(tmp_path / "engine.snap")
    a.snapshot(path)
    b = d.Engine(0)
    b.resume(path)
    for x, y in zip(a.export_graph(), b.export_graph()):
        assert np.array_equal(x, y)
    for i in range(half, len(ups), 256):
        ra, rb = a.run_batch(ups[i:i + 256]), b.run_batch(ups[i:i + 256])
        assert ra.batch_id == rb.batch_id
        assert ra.qids.tolist() == rb.qids.tolist() == [ids[0], ids[2]]
        assert np.array_equal(ra.signs, rb.signs) and np.array_equal(ra.counts, rb.counts)
        assert np.array_equal(ra.tuples, rb.tuples)
    with pytest.raises(d.DSMError):
        b.resume(path)  # queries are registered now
    a.close()
    b.close()
