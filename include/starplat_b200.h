/* starplat_b200 — C ABI of the B200-native (sm_100a) static-graph kernels.
 *
 * Drop-in boundary: StarPlat's code generators emit one C++ entry point per DSL
 * program, taking the CSR container `graph&` plus raw property arrays
 * (signature emitter: src/backends/backend_omp/dsl_cpp_generator.cpp:3098-3151,
 * type mapping :2875-3050). include/starplat_b200.hpp keeps those exact C++
 * signatures and forwards to the plain-pointer functions below.
 *
 * Conventions
 *   - Every function returns an int status: SP_OK (0) or a negative SP_ERR_*;
 *     sp_last_error() gives a message for the calling thread. No exceptions
 *     cross this ABI.
 *   - Array arguments may be host or device pointers (CUDA unified addressing
 *     decides the copy direction). Output arrays are sized num_nodes().
 *   - A graph handle is used from one host thread at a time.
 *   - All indices are int32, as in graph.hpp:44-57; edge counts must be < 2^31.
 */
#ifndef STARPLAT_B200_H
#define STARPLAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SP_OK = 0,
  SP_ERR_INVALID = -1,     /* bad argument or malformed CSR */
  SP_ERR_CUDA = -2,        /* CUDA runtime error */
  SP_ERR_OOM = -3,         /* device allocation failed */
  SP_ERR_TIMEOUT = -4,     /* a bounded device-side loop ran out of iterations */
  SP_ERR_UNSUPPORTED = -5, /* input outside what this build handles */
  SP_ERR_NEG_CYCLE = -6    /* SSSP: negative cycle reachable from the source */
};

typedef struct sp_graph* sp_graph_h;

/* graph creation flags */
#define SP_GRAPH_DEVICE_PTRS 0x1u  /* the CSR pointers given are device pointers */

/* ---- library -------------------------------------------------------------- */
int sp_version(void);
const char* sp_last_error(void);
/* Number of kernels this library has launched in this process (graph nodes count once each). */
unsigned long long sp_launch_count(void);
/* Device memory released by this library (graph handles, plans, scratch) is kept in a
 * per-device cache, at most 1/8 of the device's memory or 4 GiB, and reused by later
 * allocations of a similar size. sp_cache_bytes: bytes held for the current device.
 * sp_cache_trim: returns every cached block to the driver (like
 * torch.cuda.empty_cache); an allocation that runs out of memory does the same for
 * its device before failing. bytes_freed may be NULL. */
int sp_cache_bytes(int64_t* bytes);
int sp_cache_trim(int64_t* bytes_freed);

/* ---- device mirror of graph.hpp's CSR (uploaded once, reused by every call) ----
 * Replaces the per-call H2D copy of the generated CUDA code
 * (backend_cuda/dsl_cpp_generator.cpp:4104-4297, generateCSRArrays).
 * indexofNodes[V+1], edgeList[E]: forward CSR (graph.hpp:44-50), adjacency sorted.
 * edgeLen[E] (weights, graph.hpp:38) may be NULL.
 * rev_indexofNodes[V+1], srcList[E] (graph.hpp:45-52) may be NULL: then the
 * reverse CSR is built on the device. */
int sp_graph_create(int32_t V, int64_t E, const int32_t* indexofNodes, const int32_t* edgeList,
                    const int32_t* edgeLen, const int32_t* rev_indexofNodes, const int32_t* srcList,
                    uint32_t flags, sp_graph_h* out);
int sp_graph_free(sp_graph_h g);
/* Builds the device mirror straight from a text edge list, in place of
 * graph::parseGraph (graph.hpp:464-512 parseEdges, :720-865 parseEdgesContent): one
 * edge per line "src dst weight"; lines that are empty or do not start with a digit
 * are skipped; fields are read as std::stringstream reads integers (sign, digits up
 * to the first other character; a malformed weight reads 0); V = largest id + 1;
 * duplicate pairs become one edge with the summed weight; self-loops are kept. Where
 * the reference is undefined: a line without a weight gets weight 1, and a missing,
 * malformed, negative or out-of-range id is SP_ERR_INVALID naming the line.
 * Host threads tokenise (nthreads <= 0: all cores); sorting, merging and both CSRs
 * are built on the device. */
int sp_graph_load_text(const char* path, int32_t nthreads, sp_graph_h* out);
/* Copies the mirror's CSR to host buffers, each optional (NULL skips it), sized like
 * the reference's fields: indexofNodes[V+1], edgeList[E], edgeLen[E],
 * rev_indexofNodes[V+1], srcList[E], edgeMap[E] (edgeMap[i] = forward index of
 * reverse entry i, graph.hpp:836-846; built on the first request). V and E come
 * from sp_graph_info. */
int sp_graph_export(sp_graph_h g, int32_t* indexofNodes, int32_t* edgeList, int32_t* edgeLen,
                    int32_t* rev_indexofNodes, int32_t* srcList, int32_t* edgeMap);
/* Replaces graph::updateCSRDel / updateCSRAdd (graph.hpp:869-980) for one batch of n
 * updates, the fields of the reference's `update` record (update.hpp:9-16) as host
 * arrays: type[i] 'd' (delete) or 'a' (add), src[i] -> dst[i], weight[i] (NULL = 1).
 * As a DSL Batch block does, the deletions apply first, then the additions. Deleting a
 * missing edge does nothing; adding an edge that is present sums its weights (the
 * parseGraph rule for duplicates), where the reference's diff-CSR would keep two edges.
 * The vertex count stays V; an id outside [0, V) or another type rejects the whole
 * batch with SP_ERR_INVALID and leaves g unchanged. The forward CSR is rebuilt on the
 * device (one sort of the old and added edge keys); the reverse CSR, edgeMap and every
 * algorithm's plan are rebuilt on the next call that needs them. A graph without
 * edgeLen stays without. */
int sp_graph_update(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                    const int32_t* weight);
/* Use this CUDA stream (a cudaStream_t) for all later work on g; NULL = the library's own
 * stream (the one every graph starts with: a blocking stream, so it is ordered with work on
 * the legacy default stream). To run on the legacy default stream itself pass
 * cudaStreamLegacy, not NULL. */
int sp_graph_set_stream(sp_graph_h g, void* cuda_stream);
/* V, E, symmetric (1 when the forward CSR equals the reverse CSR). */
int sp_graph_info(sp_graph_h g, int32_t* V, int64_t* E, int32_t* symmetric);

/* Schedule knobs (what the autotuner and the learned scheduler set); results never
 * depend on them. Unknown keys: SP_ERR_INVALID.
 *   "pr.hot"  PageRank: source ids (after relabelling by out-degree) gathered in the
 *             L1-resident hot phase of each iteration (0..2^22, default 0 = one phase
 *             for all sources).
 *   "pr.src_hint"  PageRank: L1 policy of the srcList loads, read once per iteration
 *             (0 cached, 1 not allocated, 2 evicted first = default).
 *   "pr.order"  PageRank vertex order, fixed when the plan is built (a change rebuilds
 *             it): 0 = out-degree descending; 1 = in-degree class first (the row bins
 *             of the iteration kernel), out-degree descending within a class.
 *   "pr.l1_hot"  PageRank: only gathers from the first l1_hot sources (relabelled by
 *             out-degree, so the most-gathered ones) allocate in L1; the others bypass
 *             it (0..2^22, default 32768; 0 = every gather allocates).
 *   "pr.vec"  PageRank: 1 = the 32-lane bin and the long-row chunks read srcList in
 *             16-byte loads (four entries per lane), 0 = one entry per lane per load.
 *   "sssp.delta"  SSSP bucket width used when sp_sssp gets delta <= 0 (0 = the largest
 *             edge weight).
 *   "sssp.ctas_per_sm"  SSSP: persistent CTAs per SM of the delta-stepping kernel (1..8,
 *             default 4; fewer CTAs make each grid barrier cheaper on high-diameter graphs).
 *   "sssp.batch"  sp_sssp_batch / sp_closeness: sources per cooperative launch, each on
 *             its own group of CTAs (1..1024, default 4; capped by the co-resident CTAs
 *             and by 1/8 of device memory at 44 bytes per vertex per source).
 *   "sssp.last_batch" (read only): sources per launch of the last batched run.
 *   "sssp.last_delta", "sssp.last_ctas", "sssp.last_local" (read only): the schedule the
 *             last SSSP call ran; "sssp.last_relaxed": the edges it relaxed (each
 *             out-edge of a vertex once per time the vertex was expanded).
 *   "tc.cta_warps"  TC on graphs of up to 65536 vertices: 0 = a bitmap per warp;
 *             2, 4, 8 or 16 = one bitmap per CTA of that many warps sharing each anchor.
 *   "tc.last_incremental" (read only): 1 if the last sp_tc_dynamic counted only the
 *             triangles through the batch's edges, 0 if it counted the graph again.
 *   "sssp.hub_deg", "sssp.hub_chunk"  SSSP: queued vertices with more out-edges than
 *             hub_deg are relaxed in hub_chunk-edge pieces shared by all warps
 *             (defaults 128 and 64).
 *   "sssp.repair"  sp_sssp_dynamic: 1 = a batch with deletions repairs through parents
 *             (weights >= 1), 0 = it solves again from the source, -1 (default) = repair
 *             when the graph's last solve from a source took at least 32 rounds. The
 *             repair pays on high-diameter graphs (grid 1024^2, 64 deletions: 1.5 ms
 *             against 8.3 ms for update + solve) and loses where a solve takes a dozen
 *             rounds (R-MAT 20: 3.4 against 2.2 ms). "sssp.last_marked" (read only):
 *             vertices the last repair reset (-1: no repair ran).
 *   "sssp.filter"  SSSP: 1 = load dist[u] and send the atomicMin only when the candidate
 *             is lower; 0 = send every atomicMin at once (one L2 round trip less per
 *             hop, more atomics); -1 = default: 0 inside warp cascades, 1 elsewhere.
 *   "sssp.local"  SSSP: in rounds whose frontier is at most 32 vertices per warp, a warp
 *             keeps relaxing the vertices it improved below the bucket threshold, up to
 *             this many 32-edge steps per round, before the grid barrier (0 = off,
 *             default 64). Unset, the learned scheduler chooses between 0 and 64.
 *   "bc.hub_deg", "bc.hub_chunk"  BC: level-list entries of vertices with more than
 *             hub_deg edges are cut into hub_chunk-edge pieces shared by all warps
 *             (defaults 64 and 64).
 *   "bc.batch"  BC: sources traversed together in one multi-source pass (1..64, default 64).
 *   "bc.dir"  BC forward direction per level (one cooperative launch, sp_bc and
 *             sp_bfs_sigma): 0 push (expand the level's entries along out-edges);
 *             1 pull while bc.pull_alpha * (out-edges of the level's entries) exceeds the
 *             in-edges of the vertices some source has not reached + V / 8 (pull: every
 *             such vertex scans its in-edges for parents in the level, no atomics except
 *             on vertices above 1024 in-edges); 2 a seeded random direction per level
 *             ("bc.dir_seed", exploration); 3 pull at every level; 4 the level model
 *             (sp_sched_level_load) scores push and pull from the level's statistics
 *             (rule 1 without a model). Default: 4 when a level model is loaded, else 0.
 *             The decision is taken on the device from counters every CTA reads after the
 *             same barrier, so every CTA takes the same direction.
 *   "bc.pull_alpha"  factor of the bc.dir = 1 rule, in thousandths (default 1000).
 *   "bc.trace"  1: record per level (entries, their out-edges, unreached in-edges, pull)
 *             and the device timer; read with sp_bc_level_trace.
 *   "bc.cluster"  BC of many graphs (sp_bc_graphs): CTAs per graph, 1 (default), 2, 4 or 8;
 *             above 1 the CTAs of a thread-block cluster share a graph and synchronise with
 *             hardware cluster barriers. */
int sp_tune_set(sp_graph_h g, const char* key, int64_t value);
int sp_tune_get(sp_graph_h g, const char* key, int64_t* value);

/* ---- triangle counting -------------------------------------------------------
 * Replaces generated `auto Compute_TC(graph& g)` (DSL staticDSLCodes/triangle_counting_dsl:1-13):
 *   count = sum_v sum_{u in N(v), u<v} sum_{w in N(v), w>v} [u->w is an edge]
 * Exact int64. SP_TC_TUNED: undirected graphs use a degree-ordered orientation
 * and warp-cooperative hash intersection; other graphs follow the formula
 * literally. SP_TC_PLAIN: the generated CUDA form (one thread per vertex, binary
 * search per pair; libcuda.cuh:187-212). */
#define SP_TC_TUNED 0
#define SP_TC_PLAIN 1
int sp_tc(sp_graph_h g, int64_t* triangle_count, int32_t variant);

/* ---- clustering coefficient ---------------------------------------------------
 * Replaces generated `void staticClusteringCoeff(graph& g, int* cf)` (DSL
 * staticDSLCodes/clustering_coeff:1-14): the Compute_TC loop, where every triangle
 * (v, u, w) it finds adds one to cf of all three vertices. On a symmetric graph cf[v]
 * is the number of triangles through v. cf[V] (int32, host or device) is overwritten.
 * SP_TC_TUNED: the triangle-counting kernels with per-vertex counts; SP_TC_PLAIN: the
 * generated CUDA form (one thread per vertex, binary search per pair). Exact. */
int sp_clustering_coeff(sp_graph_h g, int32_t* cf, int32_t variant);

/* ---- triangle counting over several GPUs --------------------------------------
 * For one process per GPU, each holding the whole graph (the TC graphs are small:
 * R-MAT 16 is 7 MB): part `part` of `nparts` (0 <= part < nparts) counts only the
 * triangles anchored at every nparts-th vertex of the tuned kernels' heaviest-first
 * anchor order, starting at position part. Every triangle falls in exactly one part,
 * so the parts' counts sum to sp_tc's and their cf vectors to sp_clustering_coeff's
 * (one all-reduce of an int64, or of int32[V]). Exact. nparts = 1 is the whole graph.
 * The reference's multi-GPU generator splits every forall into contiguous vertex
 * ranges (backend_multigpu/dsl_cpp_generator.cpp:4286-4288); the strided order keeps
 * the parts' work even on skewed degrees. cf[V] is overwritten. */
int sp_tc_part(sp_graph_h g, int32_t part, int32_t nparts, int64_t* triangle_count);
int sp_clustering_coeff_part(sp_graph_h g, int32_t part, int32_t nparts, int32_t* cf);

/* ---- degree and closeness centrality -----------------------------------------
 * Replaces generated `void Degree(graph& g, int* deg)` (DSL
 * staticDSLCodes/degree_centrality:1-6): deg[v] = out-degree of v. */
int sp_degree_centrality(sp_graph_h g, int32_t* deg);
/* Replaces generated `void Compute_CC(graph& g, float* CC, std::set<int>& sourceSet)`
 * (DSL staticDSLCodes/CC:1-26): CC[src] = 1.0 / (sum of the finite shortest-path
 * distances from src over the edge weights) for every source, CC = 0 elsewhere.
 * weight NULL = the graph's edgeLen. Distances by the batched solve of sp_sssp_batch
 * (learned schedule); the sum is exact in 64 bits, where the DSL's int would overflow
 * past 2^31 - 1. Sources must be distinct; CC[V] host or device. */
int sp_closeness(sp_graph_h g, const int32_t* weight, const int32_t* sources, int32_t nsrc, float* CC);
/* Replaces generated `void Compute_CC_Unweighted(graph& g, float* CC, std::set<int>& sourceSet)`
 * (DSL staticDSLCodes/closeness_centrality_unwt:1-20): CC[src] = 1.0 / (sum of the BFS
 * levels of the vertices reached from src), CC = 0 elsewhere. Levels from the batched
 * BFS of sp_bc, 64 sources per pass. */
int sp_closeness_unweighted(sp_graph_h g, const int32_t* sources, int32_t nsrc, float* CC);

/* ---- PageRank ----------------------------------------------------------------
 * Replaces generated `void ComputePageRank(graph& g, float beta, float delta, int maxIter,
 * float* pageRank)` (DSL staticDSLCodes/PageRankDSLV3:1-25): Jacobi pull over the
 * reverse CSR, pr0 = 1/V, pr' = (1-delta)/V + delta * sum pr[u]/outdeg(u), repeated
 * while L1 diff > beta and iterations < maxIter. FP32 ranks, FP64 row sums.
 * iterations / final_diff may be NULL. variant: SP_PR_TUNED or SP_PR_PLAIN. */
#define SP_PR_TUNED 0
#define SP_PR_PLAIN 1
int sp_pagerank(sp_graph_h g, float beta, float delta, int32_t maxIter, float* pageRank,
                int32_t* iterations, double* final_diff, int32_t variant);

/* PageRank split over the GPUs of a node by vertices, one part per rank; replaces the
 * host-staged copies of the reference's multi-GPU generator
 * (backend_multigpu/dsl_cpp_generator.cpp:604-678). Every rank holds the whole graph
 * and owns the rows of one part; the caller's collectives run between the calls, on
 * the same stream (sp_graph_set_stream), with device buffers:
 *   begin    part in [0, nparts); con0 / con1: the caller's ping-pong contrib buffers,
 *            DEVICE, nparts * S floats each; diff: one DEVICE double; *slice = S.
 *   iterate(k), k = 0, 1, ...: the part's rows of iteration k: reads con[k % 2], writes
 *            the part's block con[(k + 1) % 2][part * S, (part + 1) * S) and its L1 diff
 *            into *diff. The caller then all-gathers the blocks of con[(k + 1) % 2]
 *            (equal S-float blocks, in part order) and sums *diff over the ranks.
 *   decide   the stop test on the summed diff (diff > beta and fewer than maxIter
 *            iterations: go on), on the device; later iterate calls of a finished run
 *            return at once, so a caller may queue several iterations before it reads
 *            the state (one synchronisation per several iterations).
 *   state    iterations run, done flag and the last summed diff (synchronises).
 *   ranks    the part's S ranks (its block, in the split plan's order) into slice,
 *            host or device; the caller all-gathers them into nparts * S floats.
 *   finish   that gathered DEVICE vector to pageRank[V] in the caller's vertex order.
 * With the same beta, delta and maxIter every rank reaches the ranks of sp_pagerank to
 * FP32 rounding of the per-row FP64 sums. */
int sp_pagerank_part_begin(sp_graph_h g, int32_t part, int32_t nparts, float beta, float delta, int32_t maxIter,
                           float* con0, float* con1, double* diff, int32_t* slice);
int sp_pagerank_part_iterate(sp_graph_h g, int32_t k);
int sp_pagerank_part_decide(sp_graph_h g);
int sp_pagerank_part_state(sp_graph_h g, int32_t* iterations, int32_t* done, double* diff);
int sp_pagerank_part_ranks(sp_graph_h g, float* slice);
int sp_pagerank_part_finish(sp_graph_h g, const float* ranks, float* pageRank);

/* ---- single-source shortest paths --------------------------------------------
 * Replaces generated `void Compute_SSSP(graph& g, int* dist, int* weight, int src)`
 * (DSL staticDSLCodes/sssp_dslV3:1-26). weight[E] in forward-CSR order (the drivers
 * fill it that way, main_functions/sssp_dslv2main.cpp:33-41); NULL = the graph's edgeLen.
 * dist[v] = exact shortest distance, INT_MAX when unreachable. Negative weights are
 * allowed without negative cycles (SP_ERR_NEG_CYCLE otherwise).
 * SP_SSSP_DELTA: delta-stepping in one persistent kernel; delta <= 0 picks the tuned /
 * default bucket width. SP_SSSP_PLAIN: the generated code's topology-driven form.
 * rounds (may be NULL) receives the number of relaxation rounds. */
#define SP_SSSP_DELTA 0
#define SP_SSSP_PLAIN 1
int sp_sssp(sp_graph_h g, const int32_t* weight, int32_t src, int32_t* dist, int64_t delta, int32_t variant,
            int32_t* rounds);
/* Shortest paths from many sources, for callers of the generated Compute_SSSP body in
 * a loop over sources (the per-source fixedPoint of staticDSLCodes/CC:7-19): the
 * sources run in batches of "sssp.batch", each batch ONE cooperative launch in which
 * every source has its own group of CTAs (group barriers, its own queues) and the
 * schedule is the one sp_sssp would use on this graph. dist[nsrc * V], source-major
 * (row k = distances from sources[k]), host or device; sources in [0, V), host or
 * device. Distances are bit-identical to sp_sssp's. */
int sp_sssp_batch(sp_graph_h g, const int32_t* weight, const int32_t* sources, int32_t nsrc, int32_t* dist);

/* Single-source SSSP split over GPUs by vertices: the 1-D partition with a per-bucket
 * frontier exchange, in place of the host-staged property copies of the reference's
 * multi-GPU generator (backend_multigpu/dsl_cpp_generator.cpp:604-678, :964-1005). Every
 * rank holds the whole graph and owns the vertices v with v % nparts == part. The caller
 * runs the collectives between the calls, on the same stream (sp_graph_set_stream),
 * on DEVICE buffers:
 *   begin     weight as in sp_sssp; delta <= 0 = the schedule sp_sssp would choose;
 *             *cap = ceil(V / nparts). send and recv hold nparts * cap pairs of int32.
 *   loop over rounds:
 *     relax   the part's frontier: send <- (vertex, distance) pairs for the other parts'
 *             vertices, packed in part order, send_counts[nparts] pairs each (at most
 *             one pair per vertex per round).
 *             The caller all-to-alls the counts, then the pairs.
 *     apply   the n received pairs (msgs); *frontier = this part's next frontier size.
 *             The caller sums *frontier over the ranks; while the sum is > 0, relax again.
 *     far_min when the sum is 0: *far_min = this part's smallest far distance (INT_MAX:
 *             none). The caller takes the minimum over the ranks: INT_MAX ends the solve.
 *     advance otherwise: the next bucket from the global *far_min; *frontier as in apply
 *             (sum it, then relax again).
 *   dist      dist[V] (host or device): the owned entries, INT_MAX elsewhere; the
 *             minimum over the ranks is Compute_SSSP's dist.
 * Negative weights run as one bucket; more than 4V + 64 rounds is SP_ERR_NEG_CYCLE
 * (from apply). A message for a vertex the part does not own is SP_ERR_INVALID. */
int sp_sssp_part_begin(sp_graph_h g, int32_t part, int32_t nparts, const int32_t* weight, int32_t src,
                       int64_t delta, int32_t* cap);
int sp_sssp_part_relax(sp_graph_h g, int32_t* send, int32_t* send_counts);
int sp_sssp_part_apply(sp_graph_h g, const int32_t* msgs, int32_t n, int32_t* frontier);
int sp_sssp_part_far_min(sp_graph_h g, int32_t* far_min);
int sp_sssp_part_advance(sp_graph_h g, const int32_t* far_min, int32_t* frontier);
int sp_sssp_part_dist(sp_graph_h g, int32_t* dist);

/* ---- betweenness centrality ----------------------------------------------------
 * Replaces generated `void Compute_BC(graph& g, float* BC, std::set<int>& sourceSet)`
 * (DSL staticDSLCodes/bc_dslV2:1-21): Brandes over the given distinct sources,
 * BC[v] = sum over sources s != v of the dependency delta_s[v] (no halving, as the
 * generated code). sigma is FP64 (exact below 2^53), dependencies FP32 stored /
 * FP64 summed, BC accumulated in FP64 and written as float.
 * SP_BC_BATCHED: multi-source traversal, 64 sources per pass, one persistent launch.
 * SP_BC_PLAIN: one source at a time, one thread per vertex per level (the manual /
 * generated CUDA form). */
#define SP_BC_BATCHED 0
#define SP_BC_PLAIN 1
int sp_bc(sp_graph_h g, const int32_t* sources, int32_t nsrc, float* BC, int32_t variant);

/* The forward half of the same multi-source pass: BFS levels (-1 = unreached) and
 * shortest-path counts (FP64) from up to 64 distinct sources, written source-major:
 * level[k*V + v], sigma[k*V + v]. Same level-synchronous BFS the generated code runs
 * (backend_omp/dsl_cpp_generator.cpp:64-193) with sigma of bc_dslV2:8-11. */
int sp_bfs_sigma(sp_graph_h g, const int32_t* sources, int32_t nsrc, int32_t* level, double* sigma);

/* Many independent graphs stored as one graph whose vertex ranges
 * [vertex_offset[k], vertex_offset[k+1]) have no edges between them; graph k's
 * sources are sources[source_offset[k] .. source_offset[k+1]) (global ids).
 * BC[V] gets every graph's centrality. One persistent launch, one CTA per graph
 * (largest first), no per-graph host round trip. No counterpart in the generated
 * code (it handles one graph per call); the per-graph result equals sp_bc on that
 * graph alone. */
int sp_bc_graphs(sp_graph_h g, int32_t ngraphs, const int32_t* vertex_offset, const int32_t* source_offset,
                 const int32_t* sources, float* BC);

/* ---- Louvain community detection -----------------------------------------------
 * DSL staticDSLCodes/community_detection:1-211 (MPI-only in the reference; its
 * generated entry point would be `auto Compute_CD(graph& g, int* weight)` returning
 * the modularity). weight[E] in forward-CSR order, NULL = unit weights. Local moves
 * and aggregation repeat while modularity improves by more than `threshold`
 * (the DSL uses 1e-4). community (may be NULL) gets a dense community id per vertex;
 * *modularity the final Q; levels / sweeps (may be NULL) the number of levels and
 * of local-move sweeps run.
 * SP_LV_TUNED: degree-binned warp / CTA kernels with shared-memory hash tables.
 * SP_LV_PLAIN: one thread per vertex, each candidate community's weight found by
 * rescanning the neighbour list (the O(deg^2) shape of the reference's runnable CUDA
 * Louvain, communitydetection_sequential_allocation.cu moveNodesKernel). Both use the
 * same gains and tie-breaks: with integer weights they return the same partition. */
#define SP_LV_TUNED 0
#define SP_LV_PLAIN 1
int sp_louvain(sp_graph_h g, const float* weight, double threshold, int32_t* community, double* modularity,
               int32_t* levels, int32_t* sweeps, int32_t variant);

/* ---- learned scheduler ----------------------------------------------------------
 * No counterpart in the reference. A small MLP scores candidate schedules (for SSSP:
 * bucket width, CTAs per SM and warp cascades on or off) from graph features and
 * predicts their log run time;
 * sp_sssp with delta <= 0 and no "sssp.delta" knob runs the best-scored candidate when
 * a model is loaded, else the fixed heuristic. Schedules never change results.
 * Network: x[SP_MLP_IN] -> tanh(H) -> tanh(H) -> 1, H = SP_MLP_HIDDEN, parameters
 * W1(H x IN) b1 W2(H x H) b2 w3 b3 in that order (SP_MLP_PARAMS floats). Host or device
 * pointers. sp_mlp_grad: gradient of the mean squared error (for checking against a
 * CPU reference); sp_mlp_train: full-batch Adam, all steps in one fused launch. */
#define SP_MLP_IN 13
#define SP_MLP_HIDDEN 32
#define SP_MLP_PARAMS (SP_MLP_HIDDEN * SP_MLP_IN + SP_MLP_HIDDEN * SP_MLP_HIDDEN + 3 * SP_MLP_HIDDEN + 1)
int sp_mlp_forward(const float* params, const float* X, int32_t N, float* y);
int sp_mlp_grad(const float* params, const float* X, const float* T, int32_t N, float* grad, float* loss);
int sp_mlp_train(float* params, const float* X, const float* T, int32_t N, int32_t steps, float lr, float* final_loss);
/* Load (params != NULL) or unload (params == NULL) the process-wide scheduling model;
 * feat_mean/feat_scale normalise inputs: x' = (x - mean) * scale. */
int sp_sched_load(const float* params, const float* feat_mean, const float* feat_scale);
/* No counterpart in the reference (the learned per-iteration schedule). Load or unload
 * the process-wide SSSP epoch model: the same network shape, scoring for every bucket
 * advance of a delta-stepping solve each width factor (1/4, 1/2, 1, 2, 4, 8 times the
 * call's delta) from inputs the kernel computes on the device (far-pile size, rounds
 * and relaxations of the previous epoch, progress, the previous factor, graph shape);
 * the kernel takes the factor with the lowest predicted log cost per unit of distance.
 * Knob "sssp.epoch": -1 (default) learned when a model is loaded, else fixed width;
 * 0 fixed; 1 learned; 2 a seeded pseudo-random factor per epoch ("sssp.epoch_seed",
 * exploration). Knob "sssp.epoch_widen" = 1 restricts the choice to factors >= 1.
 * Distances are exact under any width sequence. */
int sp_sched_epoch_load(const float* params, const float* feat_mean, const float* feat_scale);
/* No counterpart in the reference. Load or unload the process-wide BC level model: the
 * same network shape, predicting the log time of a forward level in each direction from
 * the inputs recorded by sp_bc_level_trace; with it, bc.dir defaults to 4. */
int sp_sched_level_load(const float* params, const float* feat_mean, const float* feat_scale);
/* With knob "sssp.trace" = 1 and a per-epoch policy, the last single-source solve's
 * epochs: records[k][16] = the SP_MLP_IN inputs of the chosen factor, the factor, the
 * distance the threshold advanced, padding; times[k] = device timer (ns) at advance k,
 * times[n] at the end. *n = epochs recorded; up to cap records are copied. */
int sp_sssp_epoch_trace(sp_graph_h g, float* records, unsigned long long* times, int32_t cap, int32_t* n);
/* With knob "bc.trace" = 1 and bc.dir != 0, the last sp_bc grid run's levels (over all
 * batches): records[k][16] = the level model's SP_MLP_IN inputs for the direction taken
 * (graph size, batch size, the level's entries and their out-edges, the in-edges of the
 * vertices not yet reached by every source, the level, the direction), then 1 if pulled;
 * times[k] = device timer (ns) at each level start, times[n] at the end of the run.
 * No counterpart in the reference. */
int sp_bc_level_trace(sp_graph_h g, float* records, unsigned long long* times, int32_t cap, int32_t* n);

/* ---- learned kernel variants ---------------------------------------------------
 * No counterpart in the reference, whose kernels have one fixed shape each. PageRank,
 * TC, BC and Louvain each have a table of kernel variants that change only how work is
 * split or cached (PageRank: gathers that allocate in L1, srcList policy and load width;
 * TC: the bitmap kernel's CTA width below 65537 vertices, else the hash kernel's
 * probe-list elements per lane; BC: the degree above which a level-list entry is cut
 * into shared pieces, and the piece size; Louvain: the shared-memory table size of the
 * CTA degree bin). A network of the scheduler's shape, loaded per algorithm, predicts
 * the log run time of every applicable candidate from degree statistics computed on
 * the device (PageRank, TC, BC: once per graph and model; Louvain: at every level, from
 * the level graph) and the call runs the lowest. Knob "<a>.variant" (a = pr, tc, bc,
 * lv): -1 (default) learned when a model is loaded and none of the algorithm's own
 * variant knobs is set (pr.l1_hot / pr.src_hint / pr.vec, tc.cta_warps / tc.unroll,
 * bc.hub_deg / bc.hub_chunk, lv.cta_slots), else those knobs and the defaults; -2 the
 * knobs and defaults even with a model; k >= 0 candidate k (to time the table).
 * "<a>.last_variant" (read only): the candidate the last call ran (Louvain: its last
 * level), -1 for knobs and defaults. Counts, distances, levels and path counts are the
 * same under every candidate; floating-point sums may change grouping. */
#define SP_VARIANT_PAGERANK 0
#define SP_VARIANT_TC 1
#define SP_VARIANT_BC 2
#define SP_VARIANT_LOUVAIN 3
/* Load (params != NULL) or unload (params == NULL) algo's variant model. A call leaves
 * the fixed defaults' candidate only when the best predicted log time is lower than the
 * defaults' by more than margin (>= 0; log(1.05) = a predicted gain above 5%). */
int sp_sched_variant_load(int32_t algo, const float* params, const float* feat_mean, const float* feat_scale,
                          float margin);
/* *n = the candidates in algo's table. */
int sp_variant_count(int32_t algo, int32_t* n);
/* x[SP_MLP_IN] = the inputs of candidate cand on g (BC: for a run of nsrc sources;
 * Louvain: its first level); *applicable = 0 when the candidate is not one g can run. */
int sp_variant_features(sp_graph_h g, int32_t algo, int32_t cand, int32_t nsrc, float* x, int32_t* applicable);
/* With knob "lv.trace" = 1, the last tuned sp_louvain run's levels: records[k][16] = the
 * SP_MLP_IN inputs of the candidate the level ran, its index, the level's bins, tables
 * and sweeps in device milliseconds, padding. *n = levels; up to cap records copied. */
int sp_louvain_level_trace(sp_graph_h g, float* records, int32_t cap, int32_t* n);
/* Replaces the generated Batch block of DynSSSP (DSL dynamicDSLCodes/dynamicBatchSSSP:
 * OnDelete + updateCSRDel + Decremental, then OnAdd + updateCSRAdd + Incremental): one
 * batch of edge updates as in sp_graph_update, then the distances from source on the
 * updated graph over its edgeLen. dist[V] (host or device) holds the distances from
 * source before the batch on entry (from sp_sssp or an earlier call) and after it on
 * return. A batch of additions only resumes from those distances with the sources of
 * the added edges queued: distances only drop, and each drop starts at an added edge.
 * A batch with deletions on a graph whose weights are all >= 1 repairs through parents
 * (the decremental pass): every vertex gets a parent among its tight in-edges on the old
 * graph; a record on a vertex's parent edge (deleted, or lengthened by an added weight)
 * unmarks its whole parent subtree, whose distances are reset, lowered from unmarked
 * in-neighbours, and the solve resumes from them and from the sources of the additions;
 * when the subtrees hold more than a quarter of the vertices it solves again instead.
 * Other batches with deletions, and additions to edges the graph already holds, solve
 * again from source. Results are exact on every path; the DSL's OnAdd test
 * (dest.dist > src.dist + 1) ignores the edge weight, this does not. Tune key
 * "sssp.last_incremental" (read only): 0 = solved again, 1 = resumed after additions,
 * 2 = repaired through parents. */
int sp_sssp_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                    const int32_t* weight, int32_t source, int32_t* dist);
/* Replaces the generated Batch block of DynPR (DSL dynamicDSLCodes/dynamicBatchPR:
 * OnDelete + propagateNodeFlags + updateCSRDel + Decremental, then the same for the
 * additions): one batch of edge updates as in sp_graph_update (n = 0: none), then
 * PageRank on the updated graph started from pageRank[V] (host or device; the ranks
 * before the batch, from sp_pagerank or an earlier call) instead of 1/V, with
 * sp_pagerank's iteration, stop test (L1 diff <= beta or maxIter) and outputs; the
 * new ranks are written back to pageRank. Every vertex is iterated: graph.hpp's
 * propagateNodeFlags (graph.hpp:444-462) marks the destination of every edge, so the
 * DSL's modified-only sweeps cover all vertices with in-edges, and the others hold
 * (1 - delta) / V in any PageRank output. The DSL's dynamic sweeps sum signed
 * differences (dynamicBatchPR:56); this uses the L1 sum of the static form. */
/* Replaces the generated Batch block of DynTC (DSL dynamicDSLCodes/dynamicBatchTCV2:
 * OnDelete + Decremental + updateCSRDel + updateCSRAdd + OnAdd + Incremental): one batch
 * of edge updates as in sp_graph_update, then the triangle count of the updated graph.
 * triangle_count holds sp_tc's count before the batch on entry and after it on return.
 * On a symmetric graph whose batch keeps it symmetric (deletions and additions each
 * given in both directions), only triangles through the changed edges are counted:
 * those of the old graph through edges it held and the batch deletes, and those of the
 * new graph through edges it gains, each weighted 1 / (changed edges in it). Otherwise
 * the updated graph is counted again. Exact either way; the DSL's form counts deletions
 * of absent edges and repeated updates as changes, this does not. Tune key
 * "tc.last_incremental" (read only) says which path the last call took. */
int sp_tc_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                  const int32_t* weight, int64_t* triangle_count);
/* Replaces the generated Batch block of DynCF (DSL dynamicDSLCodes/dynamicBatchClustering):
 * one batch of edge updates as in sp_graph_update, then cf[V] (host or device;
 * sp_clustering_coeff's counts before the batch on entry) brought up to date. On a
 * symmetric graph with a batch that keeps it symmetric, only the triangles through the
 * changed edges are found (as in sp_tc_dynamic), each adding -1 (deleted) or +1 (added)
 * to its three vertices once; otherwise the updated graph is counted again. Exact.
 * "tc.last_incremental" says which path the call took. */
int sp_clustering_coeff_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                                const int32_t* weight, int32_t* cf);
/* Replaces the generated Batch block of DynDegree (DSL dynamicDSLCodes/dynamicBatchDeg):
 * one batch of edge updates, then deg[V] = the out-degrees of the updated graph (the
 * DSL's per-update +1 / -1 also counts deletions of absent edges and additions of
 * present ones; these are the exact degrees). */
int sp_degree_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                      const int32_t* weight, int32_t* deg);
/* Replaces the generated Batch block of DynBC (DSL dynamicDSLCodes/dynamicDecBC,
 * dynamicBatchIncNorm, dynamicBatchDecNorm): one batch of edge updates, then BC over
 * the distinct seeds (host or device ids) on the updated graph, as sp_bc computes it.
 * Seeds are checked before the batch is applied. */
int sp_bc_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                  const int32_t* weight, const int32_t* sources, int32_t nsrc, float* BC);
int sp_pagerank_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                        const int32_t* weight, float beta, float delta, int32_t maxIter, float* pageRank,
                        int32_t* iterations, double* final_diff);
/* The SP_MLP_IN inputs the scheduler builds for SSSP on g with a candidate schedule
 * (delta multiple of the largest weight, CTAs per SM, cascade budget as for
 * "sssp.local"); weight NULL = edgeLen. */
int sp_sssp_features(sp_graph_h g, const int32_t* weight, double delta_mult, int32_t ctas_per_sm,
                     int32_t local_steps, float* x);

/* ---- PageRank without device allocation -------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc (an engine that owns all device memory through its own pool and hands
 * in its buffers, a process under a hard memory cap, a caller that cannot accept the
 * device-wide synchronisation an allocation may cause). Same semantics and tolerance
 * as sp_pagerank. All pointers are DEVICE pointers owned by the caller:
 * indexofNodes[V+1] (for out-degrees), rev_indexofNodes[V+1], srcList[E], pageRank[V].
 * Scratch is a fixed array inside the library (about 12.6 MB, held on every GPU that
 * loads the library until exit), so V is limited to SP_NOALLOC_MAX_V; larger graphs
 * get SP_ERR_INVALID. The first call on a device looks up that array's address
 * (cudaGetSymbolAddress) with the device current; make it before any stream capture.
 * The address is kept until exit: a cudaDeviceReset of that device is not supported
 * while the library is loaded. Calls share the array: calls that overlap on the GPU
 * race and must be serialised. The CSR is checked on the device before any gather
 * (offsets from 0 to E, never decreasing; srcList ids in [0, V)); a malformed graph
 * returns SP_ERR_INVALID. Each call synchronises cuda_stream before it returns.
 * cuda_stream may be NULL (default stream); iterations may be NULL. */
#define SP_NOALLOC_MAX_V (1 << 20)
int sp_pagerank_noalloc(const int32_t* indexofNodes, const int32_t* rev_indexofNodes, const int32_t* srcList,
                        int32_t V, int64_t E, float beta, float delta, int32_t maxIter, float* pageRank,
                        int32_t* iterations, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* STARPLAT_B200_H */
