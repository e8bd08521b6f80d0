"""ctypes binding of libsp_b200.so (the C ABI in include/starplat_b200.h).

The CUDA library is the only compute path: if it is missing or cannot load,
every call raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsp_b200.so")

SP_OK = 0
SP_ERR = {
    -1: "SP_ERR_INVALID",
    -2: "SP_ERR_CUDA",
    -3: "SP_ERR_OOM",
    -4: "SP_ERR_TIMEOUT",
    -5: "SP_ERR_UNSUPPORTED",
    -6: "SP_ERR_NEG_CYCLE",
}

SP_ERR_INVALID_CODE = -1
SP_GRAPH_DEVICE_PTRS = 0x1
SP_TC_TUNED = 0
SP_TC_PLAIN = 1
SP_PR_TUNED = 0
SP_PR_PLAIN = 1
SP_SSSP_DELTA = 0
SP_SSSP_PLAIN = 1
SP_BC_BATCHED = 0
SP_BC_PLAIN = 1
SP_LV_TUNED = 0
SP_LV_PLAIN = 1
SP_MLP_IN = 13
SP_MLP_HIDDEN = 32
SP_MLP_PARAMS = SP_MLP_HIDDEN * SP_MLP_IN + SP_MLP_HIDDEN * SP_MLP_HIDDEN + 3 * SP_MLP_HIDDEN + 1
SP_VARIANT_PAGERANK = 0
SP_VARIANT_TC = 1
SP_VARIANT_BC = 2
SP_VARIANT_LOUVAIN = 3

_L = None

vp = ctypes.c_void_p
i32 = ctypes.c_int32
i64 = ctypes.c_int64
f32 = ctypes.c_float
f64 = ctypes.c_double
P = ctypes.POINTER


class SPError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed: {SP_ERR.get(status, status)}: {msg}")
        self.status = status


# name -> (restype, argtypes); every symbol include/starplat_b200.h declares
SIGNATURES = {
    "sp_version": (ctypes.c_int, []),
    "sp_last_error": (ctypes.c_char_p, []),
    "sp_launch_count": (ctypes.c_ulonglong, []),
    "sp_cache_bytes": (ctypes.c_int, [P(i64)]),
    "sp_cache_trim": (ctypes.c_int, [P(i64)]),
    "sp_graph_create": (ctypes.c_int, [i32, i64, vp, vp, vp, vp, vp, ctypes.c_uint32, P(vp)]),
    "sp_graph_free": (ctypes.c_int, [vp]),
    "sp_graph_load_text": (ctypes.c_int, [ctypes.c_char_p, i32, P(vp)]),
    "sp_graph_export": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp]),
    "sp_graph_set_stream": (ctypes.c_int, [vp, vp]),
    "sp_graph_info": (ctypes.c_int, [vp, P(i32), P(i64), P(i32)]),
    "sp_graph_update": (ctypes.c_int, [vp, i64, vp, vp, vp, vp]),
    "sp_sssp_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, i32, vp]),
    "sp_tc_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, P(i64)]),
    "sp_clustering_coeff_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, vp]),
    "sp_degree_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, vp]),
    "sp_bc_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, vp, i32, vp]),
    "sp_pagerank_dynamic": (ctypes.c_int, [vp, i64, vp, vp, vp, vp, f32, f32, i32, vp, P(i32), P(f64)]),
    "sp_tune_set": (ctypes.c_int, [vp, ctypes.c_char_p, i64]),
    "sp_tune_get": (ctypes.c_int, [vp, ctypes.c_char_p, P(i64)]),
    "sp_tc": (ctypes.c_int, [vp, P(i64), i32]),
    "sp_tc_part": (ctypes.c_int, [vp, i32, i32, P(i64)]),
    "sp_clustering_coeff_part": (ctypes.c_int, [vp, i32, i32, vp]),
    "sp_pagerank": (ctypes.c_int, [vp, f32, f32, i32, vp, P(i32), P(f64), i32]),
    "sp_pagerank_part_begin": (ctypes.c_int, [vp, i32, i32, f32, f32, i32, vp, vp, vp, P(i32)]),
    "sp_pagerank_part_iterate": (ctypes.c_int, [vp, i32]),
    "sp_pagerank_part_decide": (ctypes.c_int, [vp]),
    "sp_pagerank_part_state": (ctypes.c_int, [vp, P(i32), P(i32), P(f64)]),
    "sp_pagerank_part_ranks": (ctypes.c_int, [vp, vp]),
    "sp_pagerank_part_finish": (ctypes.c_int, [vp, vp, vp]),
    "sp_sssp": (ctypes.c_int, [vp, vp, i32, vp, i64, i32, P(i32)]),
    "sp_sssp_batch": (ctypes.c_int, [vp, vp, vp, i32, vp]),
    "sp_sssp_part_begin": (ctypes.c_int, [vp, i32, i32, vp, i32, i64, P(i32)]),
    "sp_sssp_part_relax": (ctypes.c_int, [vp, vp, vp]),
    "sp_sssp_part_apply": (ctypes.c_int, [vp, vp, i32, vp]),
    "sp_sssp_part_far_min": (ctypes.c_int, [vp, vp]),
    "sp_sssp_part_advance": (ctypes.c_int, [vp, vp, vp]),
    "sp_sssp_part_dist": (ctypes.c_int, [vp, vp]),
    "sp_bc": (ctypes.c_int, [vp, vp, i32, vp, i32]),
    "sp_bc_graphs": (ctypes.c_int, [vp, i32, vp, vp, vp, vp]),
    "sp_bfs_sigma": (ctypes.c_int, [vp, vp, i32, vp, vp]),
    "sp_clustering_coeff": (ctypes.c_int, [vp, vp, i32]),
    "sp_degree_centrality": (ctypes.c_int, [vp, vp]),
    "sp_closeness": (ctypes.c_int, [vp, vp, vp, i32, vp]),
    "sp_closeness_unweighted": (ctypes.c_int, [vp, vp, i32, vp]),
    "sp_louvain": (ctypes.c_int, [vp, vp, f64, vp, P(f64), P(i32), P(i32), i32]),
    "sp_mlp_forward": (ctypes.c_int, [vp, vp, i32, vp]),
    "sp_mlp_grad": (ctypes.c_int, [vp, vp, vp, i32, vp, vp]),
    "sp_mlp_train": (ctypes.c_int, [vp, vp, vp, i32, i32, f32, vp]),
    "sp_sched_load": (ctypes.c_int, [vp, vp, vp]),
    "sp_sched_epoch_load": (ctypes.c_int, [vp, vp, vp]),
    "sp_sched_level_load": (ctypes.c_int, [vp, vp, vp]),
    "sp_sssp_epoch_trace": (ctypes.c_int, [vp, vp, vp, i32, P(i32)]),
    "sp_bc_level_trace": (ctypes.c_int, [vp, vp, vp, i32, P(i32)]),
    "sp_sssp_features": (ctypes.c_int, [vp, vp, f64, i32, i32, vp]),
    "sp_sched_variant_load": (ctypes.c_int, [i32, vp, vp, vp, f32]),
    "sp_variant_count": (ctypes.c_int, [i32, P(i32)]),
    "sp_variant_features": (ctypes.c_int, [vp, i32, i32, i32, vp, P(i32)]),
    "sp_louvain_level_trace": (ctypes.c_int, [vp, vp, i32, P(i32)]),
    "sp_pagerank_noalloc": (ctypes.c_int, [vp, vp, vp, i32, i64, f32, f32, i32, vp, P(i32), vp]),
}


def lib() -> ctypes.CDLL:
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it (python -m starplat_b200.build); "
                               "there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _L = L
    return _L


def check(fn: str, status: int) -> None:
    if status != SP_OK:
        msg = lib().sp_last_error()
        raise SPError(fn, status, msg.decode() if msg else "")


def launch_count() -> int:
    return int(lib().sp_launch_count())
