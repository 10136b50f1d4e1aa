"""Host side of the engine without a GPU: the C-ABI library loads and exports
every declared symbol; the text reader, query planner and workload generator
agree with the oracle."""
import os
import re

import numpy as np
import pytest

import dsm_b200 as d
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "dsm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dsm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = _declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(d.lib, n)]
    assert not missing, missing


def test_status_strings():
    assert d.lib.dsm_status_string(0) == b"ok"
    assert d.lib.dsm_status_string(4).startswith(b"bounded")


def test_text_reader_matches_oracle_on_fixture():
    for name, isq in (("example_q_01.in", True), ("example_g_01.in", False)):
        p = os.path.join(GOLD, name)
        a = d.TextGraph(p, isq)
        b = orc.parse(p, isq)
        assert a.nv == b["nv"] and a.ne == b["ne"]
        for k in ("labels", "offsets", "nbrs", "edges", "batch_sizes", "updates"):
            assert np.array_equal(getattr(a, k), b[k]), k


def test_text_round_trip_generated(tmp_path):
    w = d.Workload(1, scale_log2=-2)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    g = d.TextGraph(str(tmp_path / "g.in"), False)
    o = orc.parse(str(tmp_path / "g.in"), False)
    assert np.array_equal(g.edges, w.edges) and np.array_equal(g.labels, w.labels)
    assert np.array_equal(g.updates, w.updates) and np.array_equal(g.updates, o["updates"])
    assert np.array_equal(g.batch_sizes, w.batch_sizes)
    q = d.TextGraph(str(tmp_path / "q0.in"), True)
    assert np.array_equal(q.offsets, w.queries[0].offsets) and np.array_equal(q.nbrs, w.queries[0].nbrs)


def _same_graph(a, b):
    for f in ("nv", "ne"):
        assert getattr(a, f) == getattr(b, f)
    for f in ("labels", "offsets", "nbrs", "edges", "batch_sizes", "updates"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_binary_round_trip(tmp_path):
    """Text -> binary -> mapped: the same arrays as the text reader's, for a
    data file with batches and for a query file; the fixture too."""
    w = d.Workload(3, scale_log2=-8, num_batches=3)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    for src, is_q in ((tmp_path / "g.in", False), (tmp_path / "q0.in", True), (tmp_path / "q7.in", True),
                      (os.path.join(ROOT, "tests", "golden", "example_g_01.in"), False),
                      (os.path.join(ROOT, "tests", "golden", "example_q_01.in"), True)):
        out = str(tmp_path / (os.path.basename(str(src)) + ".bin"))
        d.to_binary(str(src), out, is_q)
        with open(out, "rb") as f:
            assert f.read(8) == b"DSMGRPH1"
        _same_graph(d.TextGraph(str(src), is_q), d.TextGraph(out, is_q))
        # converting the binary file again gives the same bytes
        again = out + ".2"
        d.to_binary(out, again, is_q)
        assert open(out, "rb").read() == open(again, "rb").read()


def test_binary_reader_errors(tmp_path):
    w = d.Workload(1, scale_log2=-2)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    good = str(tmp_path / "g.bin")
    d.to_binary(str(tmp_path / "g.in"), good, False)
    data = open(good, "rb").read()
    with pytest.raises(d.DSMError):  # a data graph where a query is expected
        d.TextGraph(good, True)
    cut = str(tmp_path / "cut.bin")
    open(cut, "wb").write(data[:len(data) // 2])
    with pytest.raises(d.DSMError):
        d.TextGraph(cut, False)
    bad = bytearray(data)
    nv = int.from_bytes(bad[16:20], "little")
    off0 = 64 + ((4 * nv + 63) // 64) * 64  # offsets section
    bad[off0 + 4 * 1:off0 + 4 * 2] = (2 ** 31).to_bytes(4, "little")  # offsets[1] out of order
    open(str(tmp_path / "bad.bin"), "wb").write(bytes(bad))
    with pytest.raises(d.DSMError):
        d.TextGraph(str(tmp_path / "bad.bin"), False)


def test_text_reader_errors(tmp_path):
    p = tmp_path / "bad.in"
    p.write_text("t 2 1\nv 0 0 1\nv 1 0 2\ne 0 1\n")
    with pytest.raises(d.DSMError) as e:
        d.TextGraph(str(p), True)
    assert e.value.code == 1


def test_workload_deterministic():
    a = d.Workload(1)
    b = d.Workload(1)
    assert np.array_equal(a.edges, b.edges) and np.array_equal(a.updates, b.updates)
    assert np.array_equal(a.queries[0].nbrs, b.queries[0].nbrs)
    c = d.Workload(1, seed=7)
    assert not np.array_equal(a.edges, c.edges)
    # config 1: 32768 edges, 10% withheld and re-inserted, 1000 deletions
    assert len(a.edges) == 32768 - 3276
    assert int((a.updates[:, 0] == 1).sum()) == 3276 and int((a.updates[:, 0] == 0).sum()) == 1000
    assert (a.batch_sizes == 1).all()
    assert np.array_equal(a.updates[:, 3], a.labels[a.updates[:, 1]])


def _random_connected_query(rng, nq, extra, nl):
    edges = set()
    for v in range(1, nq):
        u = int(rng.integers(0, v))
        edges.add((u, v))
    while len(edges) < nq - 1 + extra:
        a, b = sorted(int(x) for x in rng.integers(0, nq, 2))
        if a != b:
            edges.add((a, b))
    labels = rng.integers(0, nl, nq)
    perm = rng.permutation(nq)
    return d.Query.from_edges(labels, [(int(perm[a]), int(perm[b])) for a, b in sorted(edges)])


@pytest.mark.parametrize("seed", range(40))
def test_planner_matches_oracle(seed):
    """Matching orders, backward neighbours and the filter's candidacy
    positions (decycle + vertex cover + clustering) agree with the oracle."""
    rng = np.random.default_rng(seed)
    nq = int(rng.integers(2, 13))
    extra = int(rng.integers(0, nq))
    q = _random_connected_query(rng, nq, min(extra, nq * (nq - 1) // 2 - (nq - 1)), 3)
    p = d.query_plan(q)
    assert len(p["oedges"]) == int(q.offsets[-1])
    for k, (u, v) in enumerate(p["oedges"]):
        o, b = orc.order(q.offsets, q.nbrs, u, v)
        assert np.array_equal(o, p["orders"][k]) and np.array_equal(b, p["bn"][k])
    # filter positions: the oracle runs the whole filter; any data graph will do
    nv = 64
    labels = rng.integers(0, 3, nv).astype(np.uint32)
    off = np.zeros(nv + 1, np.uint32)
    _, _, pos, _ = orc.cluster_filter(q.labels, q.offsets, q.nbrs, nv, labels, off, np.zeros(0, np.uint32))
    assert np.array_equal(pos, p["enc_pos_of_u"])


def test_planner_rejects_bad_queries():
    with pytest.raises(d.DSMError):  # disconnected
        d.query_plan(d.Query.from_edges([0, 0, 0, 0], [(0, 1), (2, 3)]))
    with pytest.raises(d.DSMError):  # label beyond the signature width
        d.query_plan(d.Query.from_edges([0, 40], [(0, 1)]))
    with pytest.raises(d.DSMError):  # 17 vertices
        d.query_plan(d.Query.from_edges([0] * 17, [(i, i + 1) for i in range(16)]))
