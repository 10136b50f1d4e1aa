"""Failure path of the matcher's bounded waits, made to run out on purpose
without faulting the device.

DSM_OPT_STALL_TEST arms each matcher launch with one outstanding task that no
warp ever finishes (a flag nothing sets): once the real tasks are done every
warp waits for work, no busy warp shows progress, and each wait gives up after
DSM_OPT_TIMEOUT_MS.  The batch must then report DSM_ERR_TIMEOUT, its updates
must still be applied to the graph exactly (the graph equals the oracle's
after the batch), and the next batch with the hook off must match the oracle.
This replaces the reference's unbounded spins (queue.cuh:64-65, 84-85)."""
import time

import numpy as np
import pytest

import dsm_b200 as d
from tests.helpers import compare_batch, oracle_apply, oracle_stream, workload

pytestmark = pytest.mark.gpu

TIMEOUT = 4  # DSM_ERR_TIMEOUT
NOT_FOUND = 9


def _setup(graph=0):
    w = workload(1)
    q = w.queries[0]
    e = d.Engine(0)
    e.set_option(d.OPT_GRAPH, graph)
    e.load_graph_edges(w.nv, w.labels, w.edges)
    qid = e.register(q)
    st = oracle_stream(w.nv, w.labels, w.edges, q)
    return w, e, qid, st


def _graph_equal(e, st, tag):
    off, nb = e.export_graph()
    ooff, onb = st.export()
    assert np.array_equal(off, ooff) and np.array_equal(nb, onb), f"graph differs {tag}"


@pytest.mark.parametrize("graph", [0, 1])
def test_stalled_matcher_times_out_and_engine_recovers(graph):
    w, e, qid, st = _setup(graph)
    b1, b2, b3 = w.updates[:300], w.updates[300:600], w.updates[600:900]
    e.set_option(d.OPT_TIMEOUT_MS, 50)
    e.set_option(d.OPT_STALL_TEST, 1)
    t0 = time.perf_counter()
    with pytest.raises(d.DSMError) as ei:
        e.run_batch(b1)
    assert ei.value.code == TIMEOUT, str(ei.value)
    assert time.perf_counter() - t0 < 20.0
    st.apply_graph(b1)
    _graph_equal(e, st, "after the stalled batch")
    # an empty stalled batch still ends through the timeout
    with pytest.raises(d.DSMError) as ei:
        e.run_batch(b1[:0])
    assert ei.value.code == TIMEOUT
    e.set_option(d.OPT_STALL_TEST, 0)
    e.set_option(d.OPT_TIMEOUT_MS, 5000)
    for b in (b2, b3):
        r = e.run_batch(b)
        s, c, t, v = oracle_apply(st, b, listed=True)
        compare_batch(r, qid, s, c, t, v, tag="after recovery")
    _graph_equal(e, st, "after recovery")
    e.close()


def test_stalled_batch_in_serving_loop_reports_once():
    w, e, qid, st = _setup()
    b1, b2 = w.updates[:200], w.updates[200:400]
    e.serve_start()
    e.set_option(d.OPT_TIMEOUT_MS, 50)
    e.set_option(d.OPT_STALL_TEST, 1)
    bid = e.submit(b1)
    with pytest.raises(d.DSMError) as ei:
        e.wait(bid)
    assert ei.value.code == TIMEOUT
    with pytest.raises(d.DSMError) as ei:  # reported once, then forgotten
        e.wait(bid)
    assert ei.value.code == NOT_FOUND
    e.set_option(d.OPT_STALL_TEST, 0)
    e.set_option(d.OPT_TIMEOUT_MS, 5000)
    st.apply_graph(b1)
    r = e.results(e.submit(b2))
    s, c, t, v = oracle_apply(st, b2, listed=True)
    compare_batch(r, qid, s, c, t, v, tag="served batch after the stalled one")
    e.serve_stop()
    _graph_equal(e, st, "after serving")
    e.close()
