"""CPU: the host side of the learned kernel variants.

* the variant tables' sizes and the load/unload calls through the C ABI (no device work);
* the model files that ship with the package are well formed, and the shipped flag
  agrees with the measured decision recorded in each file;
* the margin rule that training uses to select a model (`variants._picks`) keeps the
  defaults unless a candidate is predicted faster by more than the margin.
"""
import ctypes
import json
import math
import os

import numpy as np
import pytest

from starplat_b200 import _lib, variants


def test_variant_table_sizes_through_the_c_abi():
    L = _lib.lib()
    n = ctypes.c_int32()
    sizes = {}
    for algo, code in variants.ALGOS.items():
        assert L.sp_variant_count(code, ctypes.byref(n)) == _lib.SP_OK
        sizes[algo] = n.value
    assert sizes == {"pagerank": 16, "tc": 8, "bc": 12, "louvain": 5}
    assert L.sp_variant_count(7, ctypes.byref(n)) == _lib.SP_ERR_INVALID_CODE
    # the defaults are entries of every table
    assert variants.DEFAULT_CANDIDATE["pagerank"] < sizes["pagerank"]
    assert variants.DEFAULT_CANDIDATE["bc"] < sizes["bc"]
    assert variants.DEFAULT_CANDIDATE["louvain"] == sizes["louvain"] - 1


def test_variant_model_load_checks_its_arguments():
    L = _lib.lib()
    P, IN = _lib.SP_MLP_PARAMS, _lib.SP_MLP_IN
    p = np.zeros(P, np.float32)
    mu = np.zeros(IN, np.float32)
    sc = np.ones(IN, np.float32)
    ok = L.sp_sched_variant_load(_lib.SP_VARIANT_TC, p.ctypes.data, mu.ctypes.data, sc.ctypes.data, 0.0)
    assert ok == _lib.SP_OK
    assert L.sp_sched_variant_load(_lib.SP_VARIANT_TC, None, None, None, 0.0) == _lib.SP_OK  # unload
    assert L.sp_sched_variant_load(9, p.ctypes.data, mu.ctypes.data, sc.ctypes.data, 0.0) == _lib.SP_ERR_INVALID_CODE
    assert L.sp_sched_variant_load(_lib.SP_VARIANT_TC, p.ctypes.data, None, None, 0.0) == _lib.SP_ERR_INVALID_CODE
    bad = L.sp_sched_variant_load(_lib.SP_VARIANT_TC, p.ctypes.data, mu.ctypes.data, sc.ctypes.data, -0.5)
    assert bad == _lib.SP_ERR_INVALID_CODE
    with pytest.raises(ValueError):
        variants.load_params("tc", np.zeros(P - 1, np.float32), mu, sc)


@pytest.mark.parametrize("algo", list(variants.ALGOS))
def test_shipped_model_files_are_well_formed(algo):
    path = variants.model_path(algo)
    assert os.path.exists(path), path
    d = json.load(open(path))
    assert d["algo"] == algo
    assert len(d["params"]) == _lib.SP_MLP_PARAMS
    assert len(d["feat_mean"]) == _lib.SP_MLP_IN and len(d["feat_scale"]) == _lib.SP_MLP_IN
    assert d["margin"] >= 0 and np.isfinite(d["params"]).all()
    X = np.asarray(d["X"], np.float32)
    assert X.shape == (d["samples"], _lib.SP_MLP_IN) and len(d["T"]) == d["samples"] == len(d["meta"])
    lo = d["leave_one_graph_out"]
    assert lo["learned_regret"] >= 1.0 and lo["fixed_regret"] >= 1.0
    assert isinstance(d["shipped"], bool) and d["ship_decision"].startswith("shipped" if d["shipped"] else "not shipped")
    if d["shipped"]:
        # a shipped model beat the fixed defaults on held-out graphs
        assert lo["learned_regret"] < lo["fixed_regret"]
    ev = d["evaluation"]["cases"]
    assert any(k.startswith("bench_") for k in ev) and any(k.startswith("ho_") for k in ev)


def test_only_shipped_models_load_by_default(monkeypatch):
    loaded = []
    monkeypatch.setattr(variants, "load_params", lambda a, *args, **kw: loaded.append(a))
    done = variants.load()
    shipped = [a for a in variants.ALGOS if json.load(open(variants.model_path(a))).get("shipped")]
    assert done == loaded == shipped
    loaded.clear()
    assert variants.load(shipped_only=False) == list(variants.ALGOS)


def test_margin_rule_keeps_the_defaults_unless_the_gain_is_large():
    # one graph, three candidates of PageRank's table: the defaults' entry (10), a
    # slightly faster one (predicted 3% faster) and a slower one
    meta = [("g", 10, 1.0), ("g", 0, 0.97), ("g", 3, 1.2)]
    T = np.log(np.array([1.00, 0.97, 1.20]))
    y = T.copy()  # a perfect predictor
    keep = variants._picks(y, T, meta, "pagerank", math.log(1.05))
    move = variants._picks(y, T, meta, "pagerank", 0.0)
    assert keep["g"] == pytest.approx((1.0 / 0.97, 1.0 / 0.97))  # stays on the defaults
    assert move["g"] == pytest.approx((1.0, 1.0 / 0.97))  # takes the faster entry
    # per graph, the times of its decisions are summed (Louvain: one per level)
    meta = [("h/L0", 4, 10.0), ("h/L0", 0, 5.0), ("h/L1", 4, 1.0), ("h/L1", 0, 2.0)]
    T = np.log(np.array([10.0, 5.0, 1.0, 2.0]))
    r = variants._picks(T.copy(), T, meta, "louvain", 0.0)
    assert r["h"] == pytest.approx((6.0 / 6.0, 11.0 / 6.0))
    assert variants.default_of("tc", [0, 1, 2, 3, 4]) == 2 and variants.default_of("tc", [5, 6, 7]) == 7
