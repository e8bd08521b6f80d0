"""The oracle's restatement of graph::parseGraph against the golden fixtures, which
tests/golden/make_fixtures.py made with the reference's own parseGraph (compiled from
graph.hpp); and, where this checkout has the reference build, against it directly on
fresh random files."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ANSWERS = json.load(open(os.path.join(GOLD, "known_answers.json")))


@pytest.mark.parametrize("name", sorted(ANSWERS))
def test_restatement_matches_reference_fixtures(name):
    gold = np.load(os.path.join(GOLD, "ingest", name.replace(".txt", ".npz")))
    got = O.parse_edgelist(os.path.join(GOLD, "ingest", name))
    for k in gold.files:
        assert np.array_equal(got[k], gold[k]), (name, k)
    assert got["indexofNodes"].shape[0] - 1 == ANSWERS[name]["V"]
    assert O.tc(got["indexofNodes"], got["edgeList"]) == ANSWERS[name]["tc_reference"]
    # the clustering_coeff loop's per-vertex counts, as the reference's check_if_nbr gives them
    assert O.lcc(got["indexofNodes"], got["edgeList"]).tolist() == ANSWERS[name]["lcc_reference"]


def test_reference_known_answers():
    # the reference's own fixtures: TC 3 on sample_graph.txt, TC 1 on py-starplat's input
    assert ANSWERS["sample_graph.txt"]["tc_reference"] == 3
    assert ANSWERS["py_input.txt"]["tc_reference"] == 1


def test_restatement_matches_reference_on_random_files(tmp_path):
    if O.ref_lib() is None:
        pytest.skip("reference build (oracle/_ref) not present")
    rng = np.random.default_rng(7)
    for t in range(4):
        n = int(rng.integers(1, 3000))
        s = rng.integers(0, 500, n)
        d = rng.integers(0, 500, n)
        w = rng.integers(-50, 50, n)
        p = tmp_path / f"g{t}.txt"
        p.write_text("".join(f"{a}\t{b} {c}\n" if i % 3 else f"{a} {b} {c}\r\n" for i, (a, b, c) in
                             enumerate(zip(s, d, w))))
        ref = O.ref_parse_graph(str(p))
        got = O.parse_edgelist(str(p))
        for k in ref:
            assert np.array_equal(got[k], ref[k]), (t, k)


def test_restatement_rejects_what_the_reference_leaves_undefined(tmp_path):
    for text in ("1 -3 4\n", "1\n", "5 x 2\n", "2147483647 1 1\n"):
        p = tmp_path / "bad.txt"
        p.write_text(text)
        with pytest.raises(ValueError):
            O.parse_edgelist(str(p))
    p = tmp_path / "now.txt"
    p.write_text("0 1\n1 2 \n")  # no weight field: 1 here (uninitialised in the reference)
    assert O.parse_edgelist(str(p))["edgeLen"].tolist() == [1, 1]
