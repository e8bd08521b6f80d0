"""Writes the golden fixtures under tests/golden/ from the reference compiled in this
checkout (oracle/_ref: the reference's own graph.hpp parseGraph and check_if_nbr TC
loop). Run it where the reference checkout and oracle/_ref exist:

    python tests/golden/make_fixtures.py /path/to/reference

Edge-list files (ingest/*.txt) are written by this script, except sample_graph.txt
(the reference's graphcode/sample_graphs/sample_graph.txt, as is) and py_input.txt
(py-starplat/tests/inputs/input.txt without its vertex-count header line). For every
file, ingest/<name>.npz holds the reference parseGraph arrays; files whose lines
carry no weight (the reference leaves those uninitialised) store no edgeLen.
known_answers.json holds the reference TC count of each file's graph and its
per-vertex counts of the clustering_coeff loop (the reference's check_if_nbr).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "ingest")


def write(name, lines):
    with open(os.path.join(OUT, name), "w", newline="") as f:
        f.write("".join(lines))


def main(ref_root):
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(2024)
    # 1. formatting cases: comments, blank lines, CRLF, tabs, duplicates, self-loops,
    # decimals, signs, trailing fields, sparse ids
    write("mixed.txt", [
        "# comment line\n", "% another\n", "\n", "0 1 5\n", "0\t2\t7\r\n", "1 2 3.7\n", "1 2 +4\n",
        "2 0 -2\n", "2 2 9\n", "3 1 6 extra fields\n", "  5 6 1\n", "17 3 2\n", "3 17 8\n", "0 1 5\n",
        "4 0 99999999999\n", "1 0 x\n", "9 9 1", ])
    # 2. random multigraph with duplicates and negative weights
    s = rng.integers(0, 300, 2000)
    d = rng.integers(0, 300, 2000)
    w = rng.integers(-5, 21, 2000)
    write("random_dups.txt", [f"{a} {b} {c}\n" for a, b, c in zip(s, d, w)])
    # 3. no edges at all
    write("empty.txt", ["# nothing here\n", "\n"])
    # 4. an undirected graph with known triangles (both directions listed)
    und = set()
    for _ in range(900):
        a, b = rng.integers(0, 120, 2)
        if a != b:
            und.add((int(a), int(b)))
            und.add((int(b), int(a)))
    write("undirected.txt", [f"{a} {b} {1 + (a * 7 + b * 3) % 10}\n" for a, b in sorted(und)])
    # 5. the reference's own fixtures
    with open(os.path.join(ref_root, "graphcode/sample_graphs/sample_graph.txt")) as f:
        write("sample_graph.txt", f.readlines())
    with open(os.path.join(ref_root, "py-starplat/tests/inputs/input.txt")) as f:
        write("py_input.txt", f.readlines()[1:])

    weighted = {"mixed.txt": True, "random_dups.txt": True, "empty.txt": True, "undirected.txt": True,
                "sample_graph.txt": False, "py_input.txt": True}
    answers = {}
    for name, has_w in weighted.items():
        r = O.ref_parse_graph(os.path.join(OUT, name))
        arrays = {k: v for k, v in r.items() if has_w or k != "edgeLen"}
        np.savez(os.path.join(OUT, name.replace(".txt", ".npz")), **arrays)
        answers[name] = {"V": int(r["indexofNodes"].shape[0] - 1), "E": int(r["edgeList"].shape[0]),
                         "tc_reference": int(O.ref_tc(r["indexofNodes"], r["edgeList"], 1)),
                         "lcc_reference": [int(x) for x in O.ref_lcc(r["indexofNodes"], r["edgeList"])],
                         "weights": has_w}
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(answers, f, indent=1, sort_keys=True)
    print(json.dumps(answers, indent=1))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STARPLAT_REFERENCE")
    if not root:
        sys.exit("usage: make_fixtures.py <reference checkout> (or set STARPLAT_REFERENCE)")
    main(root)
