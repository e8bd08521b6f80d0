"""GPU: sp_graph_load_text against the reference's parseGraph (golden fixtures from
graph.hpp compiled here) and against the oracle's restatement on files large enough
to split across host threads; errors name the offending line; a loaded graph runs the
algorithms like one built from the same arrays."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ANSWERS = json.load(open(os.path.join(GOLD, "known_answers.json")))


@pytest.mark.parametrize("name", sorted(ANSWERS))
def test_load_text_matches_reference_parse(name):
    gold = np.load(os.path.join(GOLD, "ingest", name.replace(".txt", ".npz")))
    with DeviceGraph.load_text(os.path.join(GOLD, "ingest", name)) as dg:
        assert (dg.V, dg.E) == (ANSWERS[name]["V"], ANSWERS[name]["E"])
        got = dg.export()
        for k in gold.files:
            assert np.array_equal(got[k], gold[k]), (name, k)
        assert dg.tc() == ANSWERS[name]["tc_reference"]
        for variant in (_lib.SP_TC_TUNED, _lib.SP_TC_PLAIN):
            assert dg.clustering_coeff(variant=variant).tolist() == ANSWERS[name]["lcc_reference"]


def _big_file(path, seed, n=150_000, V=20_000):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, V, n)
    d = rng.integers(0, V, n)
    d[: n // 10] = s[: n // 10]  # self-loops
    s[n // 2: n // 2 + n // 10] = s[: n // 10]  # duplicates
    d[n // 2: n // 2 + n // 10] = d[: n // 10]
    w = rng.integers(-9, 1000, n)
    lines = []
    for i, (a, b, c) in enumerate(zip(s, d, w)):
        if i % 997 == 0:
            lines.append("# a comment in the middle\n")
        sep = "\t" if i % 5 == 0 else " "
        end = "\r\n" if i % 7 == 0 else "\n"
        lines.append(f"{a}{sep}{b}{sep}{c}{end}" if i % 11 else f"{a} {b}{end}")  # every 11th: no weight
    with open(path, "w", newline="") as f:
        f.write("".join(lines))


def test_load_text_large_file_all_thread_counts(tmp_path):
    p = tmp_path / "big.txt"
    _big_file(p, 3)
    assert os.path.getsize(p) > (1 << 20)  # large enough to be split across threads
    ref = O.parse_edgelist(str(p))
    outs = []
    for nt in (1, 3, 8, 0):
        with DeviceGraph.load_text(str(p), nthreads=nt) as dg:
            outs.append(dg.export())
    for got in outs:
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k


def test_load_text_errors_name_the_line(tmp_path):
    p = tmp_path / "bad.txt"
    good = "".join(f"{i} {i + 1} 1\n" for i in range(100_000))
    for bad, why in (("7 -1 3\n", "destination"), ("7\n", "destination"), ("7 q 3\n", "destination"),
                     ("2147483647 1 1\n", "too large")):
        p.write_text(good + bad + good)
        with pytest.raises(_lib.SPError) as e:
            DeviceGraph.load_text(str(p), nthreads=4)
        assert ":100001:" in str(e.value) and why in str(e.value)
    with pytest.raises(_lib.SPError):
        DeviceGraph.load_text(str(tmp_path / "missing.txt"))


def test_loaded_graph_runs_like_a_built_one():
    path = os.path.join(GOLD, "ingest", "undirected.txt")
    gold = np.load(os.path.join(GOLD, "ingest", "undirected.npz"))
    with DeviceGraph.load_text(path) as a, DeviceGraph(gold["indexofNodes"], gold["edgeList"], gold["edgeLen"],
                                                       gold["rev_indexofNodes"], gold["srcList"]) as b:
        pa, ia, _ = a.pagerank(1e-6, 0.85, 100)
        pb, ib, _ = b.pagerank(1e-6, 0.85, 100)
        assert ia == ib and np.array_equal(pa, pb)
        assert np.array_equal(a.sssp(3)[0], b.sssp(3)[0])
        src = np.array([0, 5, 9], np.int32)
        assert np.array_equal(a.bc(src), b.bc(src))


def test_reverse_and_edge_map_built_on_device_for_any_graph():
    # a graph given without its reverse CSR: the stable transpose builds srcList
    # (rows ascending) and edgeMap on the device, as parseGraph does on the host
    gold = np.load(os.path.join(GOLD, "ingest", "random_dups.npz"))
    with DeviceGraph(gold["indexofNodes"], gold["edgeList"], gold["edgeLen"]) as dg:
        got = dg.export()
    for k in gold.files:
        assert np.array_equal(got[k], gold[k]), k
