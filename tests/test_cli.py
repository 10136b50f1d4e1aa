"""The CDSM command line (drop-in for DSM's `CDSM -q -d --gpu`)."""
import json
import os
import subprocess

import numpy as np
import pytest

import dsm_b200 as d
from oracle import oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_cli_usage_without_arguments():
    r = subprocess.run([d.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_cli_rejects_bad_file(tmp_path):
    p = tmp_path / "q.in"
    p.write_text("t 2 1\nv 0 0 1\nv 1 0 2\ne 0 1\n")
    r = subprocess.run([d.CLI_PATH, "-q", str(p), "-d", str(p)], capture_output=True, text=True)
    assert r.returncode == 1 and "degree" in r.stderr


def _parse(text):
    """{(batch, index): (sign, [tuples])} from CDSM output."""
    out, cur = {}, None
    for line in text.splitlines():
        f = line.split()
        if f[0] == "u":
            cur = (int(f[1]), int(f[2]))
            out[cur] = (f[6], int(f[7]), [])
        else:
            out[cur][2].append([int(x) for x in f])
    return out


@pytest.mark.gpu
def test_cli_kat_reference_fixture():
    kat = json.load(open(os.path.join(GOLD, "kat.json")))
    r = subprocess.run([d.CLI_PATH, "-q", os.path.join(GOLD, kat["query"]), "-d", os.path.join(GOLD, kat["data"]),
                        "--gpu", "0"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    res = _parse(r.stdout)
    assert res[(0, 0)][0] == "+" and res[(0, 0)][2] == kat["positive"][0]


@pytest.mark.gpu
def test_cli_generated_stream_matches_oracle(tmp_path):
    w = d.Workload(1, scale_log2=-2)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    r = subprocess.run([d.CLI_PATH, "-q", str(tmp_path / "q0.in"), "-d", str(tmp_path / "g.in"),
                        "--out", str(tmp_path / "out.txt")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    res = _parse(open(tmp_path / "out.txt").read())
    q = w.queries[0]
    st = orc.Stream(w.nv, w.labels, w.edges, q.labels, q.offsets, q.nbrs)
    signs, counts, tuples = st.apply(w.updates)
    for i in range(len(w.updates)):  # one update per batch in config 1
        sign, cnt, tup = res[(i, 0)]
        assert cnt == counts[i] and sign == {1: "+", -1: "-", 0: "0"}[int(signs[i])]
        assert np.array_equal(np.array(tup, np.uint32).reshape(-1, q.nv), tuples[i])


@pytest.mark.gpu
def test_cli_binary_inputs_equal_text(tmp_path):
    """CDSM on binary query and data files (mapped, not parsed) prints exactly
    what it prints for the text files they were converted from."""
    w = d.Workload(1, scale_log2=-2)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    d.to_binary(str(tmp_path / "q0.in"), str(tmp_path / "q0.bin"), True)
    d.to_binary(str(tmp_path / "g.in"), str(tmp_path / "g.bin"), False)
    outs = []
    for q, g in (("q0.in", "g.in"), ("q0.bin", "g.bin")):
        r = subprocess.run([d.CLI_PATH, "-q", str(tmp_path / q), "-d", str(tmp_path / g), "--gpu", "0"],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        outs.append(r.stdout)
    assert outs[0] == outs[1] and outs[0].count("\nu ") > 100


@pytest.mark.gpu
def test_cli_serve_and_graph_output_equal_plain(tmp_path):
    """--serve (every batch queued at once, merged by the serving loop) with
    --graph prints what the plain form prints, for two queries."""
    w = d.Workload(1, scale_log2=-2)
    w.write(str(tmp_path / "q"), str(tmp_path / "g.in"))
    base = [d.CLI_PATH, "-q", str(tmp_path / "q0.in"), "-d", str(tmp_path / "g.in"), "--gpu", "0",
            "--queries", str(tmp_path / "q0.in")]
    plain = subprocess.run(base, capture_output=True, text=True)
    served = subprocess.run(base + ["--serve", "--graph"], capture_output=True, text=True)
    assert plain.returncode == 0 and served.returncode == 0, served.stderr
    assert plain.stdout == served.stdout and plain.stdout.count("\nq1 u ") > 100
