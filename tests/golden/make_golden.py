"""Regenerates the golden fixtures in this folder.

Copies the reference's only test fixture (test_data/example_{q,g}_01.in of
qxk152/DSM) and writes kat.json, the known answer for its single update:
the embeddings that `a 5 6` creates, derived by hand from the query (a
triangle 0-1-2 of label 0 with a tail 1-3 (label 1), 3-4 (label 2)) and the
data graph, and the embedding counts before and after it.

    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    for name in ("example_q_01.in", "example_g_01.in"):
        shutil.copyfile(os.path.join(ref, "test_data", name), os.path.join(HERE, name))
    kat = {
        "query": "example_q_01.in",
        "data": "example_g_01.in",
        "updates": [[1, 5, 6, 0]],
        "signs": [1],
        "positive": [[[5, 6, 8, 9, 10], [5, 8, 6, 9, 10], [6, 8, 5, 9, 10], [8, 6, 5, 9, 10]]],
        "count_before": 4,
        "count_after": 8,
    }
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
