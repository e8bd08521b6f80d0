"""Golden fixtures from the reference's own runnable GPU code (test infrastructure).

Runs, on one GPU, the two GPU programs of the reference that compile from their own
sources (oracle/Makefile target `refgpu`, built where the reference checkout exists;
the binaries travel with the tree as oracle/_ref/*):

* oracle/_ref/ref_bc_manual: graphcode/manual_cuda/bcManualv5.cu. Its kernels, in the
  order BC() launches them, give the whole BC vector of each graph in BC_GRAPHS over
  its sources (the reference halves every dependency: BC += delta / 2); its unchanged
  main (parseGraph + BC(..., printAns)) prints BC[0..8] of one text graph, which pins
  the launch order of the first mode to the reference's own host code.
* oracle/_ref/ref_louvain: graphcode/dynamic_louvain_community_detection/
  communitydetection_sequential_allocation.cu, the static half of its main. For each
  graph in LOUVAIN_GRAPHS the modularity of the reference's final partition is
  computed in FP64 on the original graph (oracle.modularity, the formula of the
  reference's moveNodes, communitydetection_sequential_allocation.cu:1066-1074).

    python tests/golden/make_gpu_fixtures.py <out dir>

writes <out dir>/bc_manual.npz, bc_manual.json and louvain.json; they are committed
under tests/golden/reference_gpu/. The graphs are rebuilt by the seeded generators in
the tests, which check the stored CSR digest first.
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from starplat_b200 import generators as G  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def _weighted_sbm():
    g = G.sbm(8000, 10, seed=4)
    g.edgeLen = (1 + (G.hash_weights(g, 5, 0, 9, True) % 10)).astype(np.int32)
    return g


# name -> (graph builder, number of sources, source seed)
BC_GRAPHS = {
    "rmat12u": (lambda: G.rmat(12, 8, seed=3), 16, 3),
    "er3000": (lambda: G.erdos_renyi(3000, 10, seed=5), 16, 5),
    "grid48": (lambda: G.grid(48, 48), 8, 48),
    "rmat11d": (lambda: G.rmat(11, 8, seed=4, directed=True), 8, 4),
    "rmat16u": (lambda: G.rmat(16, 16, seed=1), 8, 16),
}
BC_TEXT_GRAPH = ("rmat10u", lambda: G.rmat(10, 8, seed=6), 8, 6)

# name -> graph builder (undirected; weighted graphs carry edgeLen)
LOUVAIN_GRAPHS = {
    "two_k5": lambda: _two_k5(),
    "grid32": lambda: G.grid(32, 32),
    "er5000": lambda: G.erdos_renyi(5000, 10, seed=3),
    "rmat12": lambda: G.rmat(12, 8, seed=2),
    "rmat16": lambda: G.rmat(16, 16, seed=1),
    "sbm20k_s1": lambda: G.sbm(20000, 24, exponent=2.0, avg_degree=32, p_in=0.8, seed=1),
    "sbm20k_s2": lambda: G.sbm(20000, 24, exponent=2.0, avg_degree=32, p_in=0.8, seed=2),
    "sbm8000_weighted": _weighted_sbm,
    "sbm1m": lambda: G.sbm(1 << 20, 256, exponent=2.0, avg_degree=32, p_in=0.8, seed=1),
}


def _two_k5():
    from starplat_b200.graph import CSRGraph

    i, j = np.triu_indices(5, 1)
    s = np.concatenate([i, i + 5]).astype(np.int32)
    d = np.concatenate([j, j + 5]).astype(np.int32)
    return CSRGraph.from_edges(10, s, d, symmetrize=True, name="2K5")


def digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.indexofNodes, np.int32).tobytes())
    h.update(np.ascontiguousarray(g.edgeList, np.int32).tobytes())
    if getattr(g, "edgeLen", None) is not None:
        h.update(np.ascontiguousarray(g.edgeLen, np.int32).tobytes())
    return h.hexdigest()[:24]


def bc_sources(g, n, seed):
    return np.sort(G.pick_sources(g, n, seed=seed)).astype(np.int32)


def run_bc_csr(g, srcs, tmp):
    inp, out = os.path.join(tmp, "g.bin"), os.path.join(tmp, "bc.bin")
    with open(inp, "wb") as f:
        f.write(np.int32(g.V).tobytes())
        f.write(np.int64(g.E).tobytes())
        f.write(np.ascontiguousarray(g.indexofNodes, np.int32).tobytes())
        f.write(np.ascontiguousarray(g.edgeList, np.int32).tobytes())
        f.write(np.int32(srcs.shape[0]).tobytes())
        f.write(np.ascontiguousarray(srcs, np.int32).tobytes())
    subprocess.run([os.path.join(REF_DIR, "ref_bc_manual"), "csr", inp, out], check=True, timeout=600)
    return np.fromfile(out, np.float64)


def run_bc_main(g, srcs, tmp):
    gp, sp = os.path.join(tmp, "g.txt"), os.path.join(tmp, "src.txt")
    G.write_edgelist(g, gp)
    with open(sp, "w") as f:
        f.write("".join(f"{int(s)}\n" for s in srcs))
    r = subprocess.run([os.path.join(REF_DIR, "ref_bc_manual"), "main", gp, sp], check=True, timeout=600,
                       capture_output=True, text=True)
    vals = {}
    for line in r.stdout.splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0].isdigit():
            vals[int(parts[0])] = float(parts[1])
    return [vals[i] for i in range(9)], r.stdout


def run_louvain(g, tmp):
    gp, cp = os.path.join(tmp, "g.txt"), os.path.join(tmp, "comm.bin")
    G.write_edgelist(g, gp, getattr(g, "edgeLen", None))
    t = time.time()
    r = subprocess.run([os.path.join(REF_DIR, "ref_louvain"), gp, cp], check=True, timeout=1800,
                       capture_output=True, text=True)
    wall = time.time() - t
    comm = np.fromfile(cp, np.int32)
    ms = float(r.stdout.split()[1]) if r.stdout.startswith("louvain_ms") else None
    return comm, ms, wall


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    bc_vec, bc_meta = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (build, n, seed) in BC_GRAPHS.items():
            g = build()
            srcs = bc_sources(g, n, seed)
            bc_vec[name] = run_bc_csr(g, srcs, tmp)
            bc_meta[name] = {"V": int(g.V), "E": int(g.E), "digest": digest(g), "sources": srcs.tolist()}
            print("bc", name, g.V, g.E, flush=True)
        name, build, n, seed = BC_TEXT_GRAPH
        g = build()
        srcs = bc_sources(g, n, seed)
        printed, _ = run_bc_main(g, srcs, tmp)
        bc_vec[name] = run_bc_csr(g, srcs, tmp)
        bc_meta[name] = {"V": int(g.V), "E": int(g.E), "digest": digest(g), "sources": srcs.tolist(),
                         "main_printed_bc_0_8": printed}
        np.savez_compressed(os.path.join(out_dir, "bc_manual.npz"), **bc_vec)
        with open(os.path.join(out_dir, "bc_manual.json"), "w") as f:
            json.dump(bc_meta, f, indent=1)
        lv = {}
        for name, build in LOUVAIN_GRAPHS.items():
            g = build()
            comm, ms, wall = run_louvain(g, tmp)
            # vertices above the file's largest id are isolated: singletons of their own
            full = np.empty(g.V, np.int32)
            full[:comm.shape[0]] = comm
            full[comm.shape[0]:] = comm.max() + 1 + np.arange(g.V - comm.shape[0])
            w = getattr(g, "edgeLen", None)
            q = O.modularity(g.indexofNodes, g.edgeList, full, None if w is None else w.astype(np.float32))
            lv[name] = {"V": int(g.V), "E": int(g.E), "digest": digest(g), "weighted": w is not None,
                        "reference_q": q, "reference_communities": int(np.unique(full).shape[0]),
                        "reference_louvain_ms": ms, "wall_s": round(wall, 1)}
            print("louvain", name, json.dumps(lv[name]), flush=True)
            with open(os.path.join(out_dir, "louvain.json"), "w") as f:
                json.dump(lv, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_gpu_fixtures.py <out dir>")
    main(sys.argv[1])
