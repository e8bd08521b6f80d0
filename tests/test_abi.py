"""CPU tests of the C ABI boundary: the library loads and exports every
function include/starplat_b200.h declares (no compute calls without a GPU)."""
import os
import re

from starplat_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sp_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_table_matches_header():
    assert declared_symbols() == set(_lib.SIGNATURES)


def test_version_and_counter():
    L = _lib.lib()
    assert L.sp_version() >= 10000
    assert _lib.launch_count() >= 0


def test_errors_do_not_cross_abi():
    import ctypes
    L = _lib.lib()
    h = ctypes.c_void_p()
    st = L.sp_graph_create(0, 0, None, None, None, None, None, 0, ctypes.byref(h))
    assert st == -1 and b"invalid" in L.sp_last_error()
    assert L.sp_graph_free(None) == 0
    assert L.sp_tc(None, None, 0) == -1


def test_dynamic_programs_slice_update_records_into_batches():
    # updates<g>.currentBatch(): consecutive slices of batchSize records, converted to the
    # C ABI's parallel arrays (host logic only; no GPU call)
    import numpy as np
    import pytest

    from starplat_b200.algorithms import _batches

    recs = [("a", 0, 1, 5), ("d", 2, 3, 0), ("a", 4, 5, 7), ("d", 6, 7, 0), ("a", 8, 9, 1)]
    got = list(_batches(recs, 2))
    assert [b[0] for b in got] == ["ad", "ad", "a"]
    assert np.array_equal(got[1][1], [4, 6]) and np.array_equal(got[1][2], [5, 7])
    assert np.array_equal(got[2][3], [1]) and got[0][1].dtype == np.int32
    assert list(_batches([], 3)) == []
    with pytest.raises(ValueError):
        list(_batches(recs, 0))
