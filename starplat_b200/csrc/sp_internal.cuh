// Internal definitions shared by the sm_100a kernels and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <utility>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/starplat_b200.h"

namespace sp {

// ----------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
extern std::atomic<unsigned long long> g_launches;  // kernels launched by this library

#define SP_CHECK_CUDA(call)                                                                  \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      ::sp::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e));     \
      return _e == cudaErrorMemoryAllocation ? SP_ERR_OOM : SP_ERR_CUDA;                     \
    }                                                                                        \
  } while (0)

#define SP_CHECK_LAUNCH()                                                                    \
  do {                                                                                       \
    ::sp::g_launches.fetch_add(1, std::memory_order_relaxed);                                \
    cudaError_t _e = cudaGetLastError();                                                     \
    if (_e != cudaSuccess) {                                                                 \
      ::sp::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(_e));      \
      return SP_ERR_CUDA;                                                                    \
    }                                                                                        \
  } while (0)

#define SP_TRY(expr)                 \
  do {                               \
    int _s = (expr);                 \
    if (_s != SP_OK) return _s;      \
  } while (0)

// ----------------------------------------------------------------- device buffer
// Device blocks come from a per-process, per-device cache (sp_graph.cu): a released
// block is kept after a device-wide synchronize (the ordering cudaFree gives) and
// handed to a later request of similar size, since cudaMalloc of a large block maps
// fresh pages and cudaFree waits for the device (each 0.2-2 ms of host time).
// dev_alloc: SP_OK, SP_ERR_OOM or SP_ERR_CUDA (message set); *got = the block's size
// (at least bytes), *dev = its device.
int dev_alloc(void** p, size_t bytes, size_t* got, int* dev);
void dev_free(void* p, size_t bytes, int dev);

template <class T>
struct dbuf {
  T* p = nullptr;
  size_t n = 0;
  size_t bytes = 0;
  int dev = 0;
  dbuf() = default;
  dbuf(const dbuf&) = delete;
  dbuf& operator=(const dbuf&) = delete;
  ~dbuf() { release(); }
  int alloc(size_t count) {
    if (count <= n && p) return SP_OK;
    release();
    const size_t b = (count ? count : 1) * sizeof(T) + 16;  // +16: vector loads may read one int4 past the end
    void* q = nullptr;
    const int st = dev_alloc(&q, b, &bytes, &dev);
    if (st != SP_OK) return st;
    p = (T*)q;
    n = count;
    return SP_OK;
  }
  void release() {
    if (p) dev_free(p, bytes, dev);
    p = nullptr;
    n = 0;
    bytes = 0;
  }
  void swap(dbuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(bytes, o.bytes);
    std::swap(dev, o.dev);
  }
};

// A view of device memory owned elsewhere (an Arena).
template <class T>
struct dspan {
  T* p = nullptr;
  size_t n = 0;
};

// Many buffers carved from one cudaMalloc. A cudaMalloc/cudaFree pair costs 0.2-0.5 ms
// of host time for large sizes (cudaFree also waits for the device), so a plan made of
// dozens of buffers asks for them with want(), then takes them all with one commit().
// Pieces start on 256-byte boundaries and carry 16 spare bytes (vector loads may read
// one int4 past the end). A later layout reuses the allocation when it fits.
struct Arena {
  dbuf<unsigned char> mem;
  size_t size = 0;
  struct Req {
    void** slot;
    size_t* n;
    size_t count, off;
  };
  std::vector<Req> reqs;
  template <class T>
  void want(dspan<T>& s, size_t count) {
    const size_t off = (size + 255) & ~(size_t)255;
    reqs.push_back({(void**)&s.p, &s.n, count, off});
    size = off + (count ? count : 1) * sizeof(T) + 16;
  }
  int commit() {
    const int st = mem.alloc(size);
    if (st != SP_OK) return st;
    for (const Req& r : reqs) {
      *r.slot = mem.p + r.off;
      *r.n = r.count;
    }
    reqs.clear();
    size = 0;
    return SP_OK;
  }
};

// ----------------------------------------------------------------- plans (per graph caches)
struct PrPlan;
struct TcPlan;
struct SsspPlan;
struct BcPlan;
struct LvPlan;
struct SsspPartPlan;
void free_pr_plan(PrPlan*);
void free_tc_plan(TcPlan*);
void free_sssp_plan(SsspPlan*);
void free_bc_plan(BcPlan*);
void free_lv_plan(LvPlan*);
void free_sssp_part_plan(SsspPartPlan*);

}  // namespace sp

// The device-resident mirror of a reference `graph` (graph.hpp:44-57).
struct sp_graph {
  int device = 0;
  int32_t V = 0;
  int64_t E = 0;
  sp::dbuf<int32_t> off;   // indexofNodes [V+1]
  sp::dbuf<int32_t> adj;   // edgeList [E]
  sp::dbuf<int32_t> w;     // edgeLen [E] (optional)
  sp::dbuf<int32_t> roff;  // rev_indexofNodes [V+1]
  sp::dbuf<int32_t> radj;  // srcList [E]
  sp::dbuf<int32_t> emap;  // edgeMap [E]: forward index of each reverse entry (built on demand)
  bool has_w = false;
  bool has_rev = false;
  int symmetric = -1;      // -1 unknown, 0/1
  int32_t max_out_deg = -1;
  int32_t pr_hot = -1;  // PageRank: source ids of the L1 hot phase (-1 = default)
  int32_t pr_order = -1;  // PageRank: vertex order of the plan (-1 = default)
  int32_t pr_src_hint = -1;  // PageRank: L1 policy of srcList loads (-1 = default)
  int32_t pr_l1_hot = -1;  // PageRank: sources whose gathers allocate in L1 (0 = all; -1 = default)
  int32_t pr_vec = -1;     // PageRank: 16-byte srcList loads (-1 = default)
  int64_t sssp_delta = 0;  // SSSP bucket width (0 = max edge weight)
  int32_t sssp_ctas_per_sm = 0;  // SSSP persistent CTAs per SM (0 = learned / 4)
  int64_t sssp_last_delta = 0;   // schedule of the last SSSP call (reporting)
  int32_t sssp_last_ctas = 0;
  int32_t sssp_last_local = 0;
  int64_t sssp_last_relaxed = 0;  // edges the last delta-stepping run relaxed
  int32_t sssp_last_incremental = 0;  // 1 if the last sp_sssp_dynamic warm-started
  int32_t tc_last_incremental = 0;    // 1 if the last sp_tc_dynamic counted only the batch
  int32_t sssp_hub_deg = 0;    // SSSP: vertices above this out-degree go to shared pieces (0 = default)
  int32_t sssp_filter = -1;    // SSSP: 1 = load dist before each atomicMin, 0 = atomicMin only (-1 = default)
  int32_t sssp_repair = -1;    // sp_sssp_dynamic: 1 = repair batches with deletions through parents, 0 = solve
                               // again, -1 = repair when the last solve took many rounds
  int32_t sssp_last_rounds = 0;  // rounds of the last delta-stepping solve from a source
  int64_t sssp_last_marked = 0;  // vertices the last repair reset (-1: no repair ran)
  int32_t sssp_hub_chunk = 0;  // SSSP: edges per piece (0 = default)
  int32_t sssp_local = -1;     // SSSP: warp cascade budget in 32-edge steps per round (-1 = default, 0 = off)
  int32_t sssp_batch = 0;      // batched SSSP: sources per cooperative launch (0 = default)
  int32_t sssp_epoch = -1;     // SSSP per-epoch width: -1 learned if an epoch model is loaded, 0 fixed, 1 learned, 2 explore
  int32_t sssp_epoch_seed = 0;  // exploration seed
  int32_t sssp_epoch_widen = 0;  // 1: the epoch model may only widen buckets
  int32_t sssp_trace = 0;      // 1: record the per-epoch trace of single-source solves
  int32_t sssp_last_epochs = 0;  // bucket advances of the last single-source solve
  int32_t sssp_last_epolicy = 0;  // the width policy the last solve ran
  int32_t sssp_last_batch = 0;  // sources per launch of the last batched run (reporting)
  int32_t tc_cta_warps = -1;  // TC: warps per CTA of the shared-bitmap kernel (-1 = default, 0 = off)
  int32_t bc_dir = -1;        // BC forward direction policy (-1 = default)
  int32_t bc_pull_alpha = 0;  // BC pull rule factor in thousandths (0 = default)
  int32_t bc_dir_seed = 0;    // BC direction exploration seed
  int32_t bc_trace = 0;       // 1: record the per-level trace of the grid form
  int32_t bc_batch = 0;
  int32_t bc_hub_deg = 0;  // BC: split level-list entries above this degree (0 = default)
  int32_t bc_hub_chunk = 0;  // BC: edges per piece of a split entry (0 = default)
  int32_t bc_cluster = 0;    // BC many-graphs form: CTAs per graph (0 = default)    // BC sources per multi-source batch (0 = 64)
  int32_t tc_unroll = -1;    // TC hash path: probe-list elements per lane per pass (-1 = default)
  int32_t lv_cta_slots = -1;  // Louvain: shared table slots of the CTA bin (-1 = default)
  int32_t lv_trace = 0;       // 1: record the per-level trace of sp_louvain
  // learned kernel variants, per algorithm (pr, tc, bc, lv): -1 learned when a variant
  // model is loaded and no variant knob is set, -2 the defaults, k >= 0 candidate k
  int32_t variant[4] = {-1, -1, -1, -1};
  int32_t last_variant[4] = {-1, -1, -1, -1};  // candidate the last call ran (-1 = knobs/defaults)
  std::vector<float> lv_trace_rec;  // per level: SP_MLP_IN inputs, candidate, ms, pad (16 floats)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  sp::PrPlan* pr = nullptr;
  sp::TcPlan* tc = nullptr;
  sp::SsspPlan* sssp = nullptr;
  sp::BcPlan* bc = nullptr;
  sp::LvPlan* lv = nullptr;
  sp::SsspPartPlan* sssp_part = nullptr;  // split single-source SSSP (sp_sssp_part_*)
};

namespace sp {
int ensure_reverse(sp_graph* g);      // builds roff/radj on device if missing
int ensure_emap(sp_graph* g);         // builds emap (edgeMap) on device if missing
// off[v] = first index of keys (ascending, E of them) that is >= v, for v = 0..V
int offsets_of_sorted(int32_t V, int64_t E, const int32_t* keys, int32_t* off, cudaStream_t s);
int finish_graph(sp_graph* g);        // checks a library-built CSR, sets max_out_deg
// one batch of edge updates on the forward CSR, deletions then additions (sp_ingest.cu);
// *held_adds (when given) receives the number of distinct added keys that were already
// edges of the graph after the deletions, whose weights grew by the added weight
int update_graph(sp_graph* g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                 const int32_t* weight, int64_t* held_adds = nullptr);
int pr_order_default();               // PageRank vertex order default (sp_pagerank.cu)
int pr_src_hint_default();
int pr_l1_hot_default();
int pr_vec_default();
int tc_cta_warps_default();           // TC kernel choice default (sp_tc.cu)
int bc_hub_deg_default();             // BC entry-splitting defaults (sp_bc.cu)
int sssp_hub_deg_default();           // SSSP hub-splitting defaults (sp_sssp.cu)
int sssp_hub_chunk_default();
int sssp_local_default();
int sssp_batch_default();         // batched SSSP sources per launch (sp_sssp.cu)
int bc_hub_chunk_default();
int bc_cluster_default();
int ensure_symmetry(sp_graph* g);     // fills g->symmetric
int copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s);  // host or device dst
// SSSP helpers shared with the split solve (sp_sssp.cu): the weights on the device (the
// caller's, host or device, or edgeLen) with their range recorded; the bucket width the
// single-GPU solve would use; the smallest weight of the last weights prepared.
int sssp_weights_for(sp_graph* g, const int32_t* weight, const int32_t** w);
int sssp_width_for(sp_graph* g, int64_t& delta);
int sssp_weight_min(sp_graph* g);
int num_sms();

// Degree statistics of a CSR (off[n+1], device), on the device: the largest row, the
// sum of squared row lengths, and for each threshold t[i] the rows longer than t[i] and
// the entries in those rows.
constexpr int DEG_THR_MAX = 6;
struct DegStats {
  int64_t max_deg = 0, sum_sq = 0;
  int64_t rows_above[DEG_THR_MAX] = {}, edges_above[DEG_THR_MAX] = {};
};
int degree_stats(const int32_t* off, int n, const int* thr, int nthr, cudaStream_t s, DegStats* out);
// The same statistics left on the device: acc[0] = largest row, acc[1] = sum of squares,
// acc[2 + 2i] / acc[3 + 2i] = rows above thr[i] / their entries (acc: 2 + 2 * DEG_THR_MAX).
int degree_stats_launch(const int32_t* off, int n, const int* thr, int nthr, unsigned long long* acc,
                        cudaStream_t s);

// Learned kernel variants (sp_mlp.cu). Algorithms index sp_graph::variant.
enum { VAR_PR = 0, VAR_TC = 1, VAR_BC = 2, VAR_LV = 3, VAR_ALGOS = 4 };
unsigned variant_generation(int algo);  // 0 = no model loaded for algo
// algo's model packed for the device (params, feature mean, scale, margin) and its
// generation (0 = none loaded, packed empty)
unsigned variant_model(int algo, std::vector<float>& packed);
// Score the rows X[k][SP_MLP_IN] with algo's model on the device; *best = the row with
// the lowest predicted log time among those with ok[k] != 0, or dflt (the fixed
// defaults' row, -1 for none) unless the best beats it by more than the model's margin.
int variant_choose(int algo, const std::vector<float>& X, const std::vector<int>& ok, int dflt, cudaStream_t s,
                   int* best);
// Per-algorithm variant tables and their inputs (in the algorithms' files).
int pr_variant_count();
int pr_variant_features(sp_graph* g, int cand, float* x, int* applicable);
int tc_variant_count();
int tc_variant_features(sp_graph* g, int cand, float* x, int* applicable);
int bc_variant_count();
int bc_variant_features(sp_graph* g, int cand, int nsrc, float* x, int* applicable);
int lv_variant_count();
int lv_variant_features(sp_graph* g, int cand, float* x, int* applicable);
}  // namespace sp

// ----------------------------------------------------------------- device helpers
namespace sp {
// The row of CSR entry x: the last vertex v in [lo, hi) with off[v] <= x, given
// off[lo] <= x < off[hi] (empty rows are never returned).
__device__ __forceinline__ int edge_source(const int32_t* __restrict__ off, int lo, int hi, long long x) {
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if (off[m] <= x) lo = m; else hi = m;
  }
  return lo;
}

// Edge-parallel loops over CSR entries: a block takes EDGE_TILE consecutive entries,
// finds the rows of the first and last by binary search over the whole offsets, and each
// thread then searches only between those two rows. Hub rows spread over many blocks.
constexpr int EDGE_TILE = 1024;

__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum with a fixed reduction tree (deterministic). All threads get the result.
template <int THREADS, class T>
__device__ __forceinline__ T block_sum(T v, T* s_red /* THREADS/32 */) {
  v = warp_sum(v);
  __syncthreads();
  if (lane_id() == 0) s_red[warp_id()] = v;
  __syncthreads();
  T r = 0;
#pragma unroll
  for (int i = 0; i < THREADS / 32; ++i) r += s_red[i];
  return r;
}
}  // namespace sp
