// Brandes betweenness centrality for sm_100a.
//
// Semantics: DSL staticDSLCodes/bc_dslV2:1-21 as emitted by the OpenMP generator
// (BFS + reverse sweep backend_omp/dsl_cpp_generator.cpp:64-193, level guard
// bfsDist[w]==bfsDist[v]+1 :1458-1495; bfsDist injected by
// SymbolTableBuilder.cpp:617-633): for every source s, a level-synchronous BFS over
// out-neighbours counts shortest paths sigma, then levels are walked backwards with
//   delta[v] = sum_{w in N(v), level(w) = level(v)+1} sigma[v]/sigma[w] * (1 + delta[w])
// and BC[v] += delta[v] for every reached v != s (the reverse loop stops at phase 1,
// so the source is excluded; no halving — the manual CUDA BC bcManualv5.cu:104
// halves, the generated code does not).
//
// B200 design — multi-source traversal (many sources share one pass over the edges):
//  * up to 32*NW sources per batch; per vertex a 64-bit mask says for which sources
//    of the batch it sits in the current frontier; sigma[v][b] (FP64, exact path
//    counts below 2^53) and delta[v][b] (FP32) are vertex-major, so the per-source
//    updates of one edge are coalesced across the warp's lanes;
//  * forward level d: lanes walk a frontier vertex's edges; q = mask & ~seen[w] are
//    the sources that reach w first at level d+1; atomicOr marks them, the first
//    marker appends w to the level list, then lanes (one per source bit) add
//    sigma with FP64 atomics (integer-valued, so the sum is exact in any order);
//  * backward level d: the masks of level d+1 are scattered into a dense array; for
//    each (v, mask) of level d the lanes pull q[w][b] = (1 + delta[w][b]) / sigma[w][b]
//    of the successors in edge order (stored in FP64 when w's dependency became final),
//    the loads of BU successors in flight together, and delta[v][b] = sigma[v][b] *
//    sum q — one 8-byte load and one add per successor instead of two loads and an FP64
//    division; no atomics, deterministic;
//  * level-list entries of vertices with more than hub_deg edges (default 64) are cut
//    into hub_chunk-edge pieces (default 64) that all warps share (one extra barrier
//    per level); their backward partials meet in an FP64 scratch through atomics;
//  * BC accumulates per vertex over the batch's sources in source order (FP64).
// One cooperative launch runs every batch of a graph (bounded grid barriers); the
// many-small-graphs form runs one CTA per graph in a persistent launch with a
// work queue (largest graphs first) and block-level barriers.
#include <cooperative_groups.h>

#include <climits>
#include <vector>

#include "sp_internal.cuh"
#include "sp_mlp_dev.cuh"
#include "sp_sync.cuh"

namespace sp {

namespace cg = cooperative_groups;

namespace bc {
constexpr int GRID_THREADS = 256;
constexpr int CTA_THREADS = 512;
// Level-list entries of vertices above HUB_DEG edges are cut into HUB_CHUNK-edge
// pieces that every warp shares. Small values balance the warps between the grid
// barriers: R-MAT 20, 256 sources: 257 ms at (4096, 256), 138 at (1024, 256),
// 121 at (128, 256), 110 at (64, 64).
constexpr int HUB_DEG = 64;
constexpr int HUB_CHUNK = 64;
constexpr int CLUSTER_DEFAULT = 1;  // CTAs per graph in the many-graphs form (bc.cluster)
// Successors whose loads are in flight together in the backward sweep (measured when
// each successor cost a sigma and a delta load),
// with the grid kernel held to 64 registers (4 CTAs per SM). R-MAT 20, 256 sources:
// 110 ms with one at a time, 87 ms with 2 at 64 registers, 97 ms with 2 at 78
// registers (3 CTAs per SM), 121 ms with 4 at 128 registers; 1000 ER graphs: 135 ->
// 104 ms.
constexpr int BU = 2;
// The same for the many-graphs kernels: with one q load per successor, 1000 ER graphs
// take 92.8 ms at 4 in flight, 126.6 ms at 2 (which spills in k_bc_graphs<1>) and
// 103.4 ms before q; R-MAT 20 (grid kernel, BU) 74.1 ms at 2, 76.7 at 4.
constexpr int BU_GRAPHS = 4;
// 32-edge chunks of one entry whose loads and atomics are in flight together in the
// forward sweep.
constexpr int FU = 2;
// Forward direction per level (knob bc.dir): 0 push only; 1 pull while
// PULL_ALPHA * (out-edges of the level) > in-edges of the vertices some source has not
// reached + V / 8 (knob bc.pull_alpha, in thousandths).
constexpr int DIR_DEFAULT = 0;
constexpr float PULL_ALPHA = 1.0f;

struct Work {
  const int32_t* __restrict__ off;  // CSR rows of this graph (global edge indices)
  const int32_t* __restrict__ adj;  // neighbour ids (subtract vbase for local ids)
  int vbase;                        // first vertex id of this graph in adj
  int V;                            // vertices of this graph
  double* sigma;                    // [V][SW]
  float* delta;                     // [V][SW]
  double* q;                        // [V][SW] (1 + delta) / sigma once delta is final: what a
                                    // predecessor's dependency sum reads of a successor
  unsigned long long* seen;         // [V]
  unsigned long long* nxt;          // [V]
  unsigned long long* dense;        // [V]
  int32_t* flv;                     // [cap] level-list vertices (local ids)
  unsigned long long* flm;          // [cap] level-list masks
  int cap;
  int* lo;                          // [maxd + 2] level starts in the lists
  int maxd;
  int* cnt;                         // append counter
  double* bc;                       // [V] FP64 accumulator (local ids)
  int* err;                         // 1 list overflow, 2 too deep, 3 barrier timeout
  // hub pieces (grid form only; hub_cap = 0 disables splitting)
  int32_t* hub_ent;                 // [hub_cap] level-list entry index
  int32_t* hub_base;                // [hub_cap] first piece index (increasing)
  unsigned long long* hub_cnt;      // (entries << 32) | pieces
  int hub_cap;
  int hub_deg;                      // entries of vertices with more edges are split
  int hub_chunk;                    // edges per piece
  double* dacc;                     // [V][SW] FP64 partial dependencies of hub entries
  // Forward direction per level (grid form): push expands the level's entries along
  // their out-edges; pull has every vertex some source of the batch has not reached scan
  // its in-edges for parents in the level (dense masks), with no atomics except on the
  // vertices of more than PULL_SPLIT in-edges, whose edges are pieces shared by all warps.
  const int32_t* __restrict__ roff;  // in-edges: the reverse CSR (off/adj when symmetric)
  const int32_t* __restrict__ radj;
  const int32_t* __restrict__ phub;  // [n_phub] vertices of more than PULL_SPLIT in-edges
  const int32_t* __restrict__ phub_base;  // [n_phub + 1] first piece of each (exclusive prefix)
  int n_phub;
  int dir_policy;                   // 0 push; 1 rule: pull while alpha * (frontier edges) > unreached edges; 2 seeded random (exploration); 3 pull whenever allowed
  float dir_alpha;
  unsigned dir_seed;
  long long e_in;                   // in-edges of the graph
  unsigned long long* ldeg;         // [maxd + 2] out-edges of each level's entries
  unsigned long long* full_in;      // in-edges of vertices every batch source has reached
  const float* dmodel;              // dir_policy 4: the level model (params, feature mean, scale)
  float* trace;                     // [trace_cap][LTRACE] per level: the chosen direction's inputs, pull
  unsigned long long* ttime;        // [trace_cap + 1] device timer at each level start, then the end
  int trace_cap;
  int* tcount;                      // levels traced
};
constexpr int PULL_SPLIT = 1024;    // in-edges per piece of a pull hub
constexpr int LTRACE = 16;          // floats per level trace record

// The inputs of the level model for direction `pull` (0 push, 1 pull) at level d with
// nent entries (values every CTA reads after the same barrier).
__device__ __forceinline__ void level_inputs(const Work& W, int d, int nent, int nsrc, int pull, float* x) {
  const float mf = (float)*(volatile unsigned long long*)(W.ldeg + d);
  const float mu = (float)((double)W.e_in - (double)*(volatile unsigned long long*)W.full_in);
  x[0] = log2f((float)W.V);
  x[1] = log2f(1.0f + (float)W.e_in);
  x[2] = (float)W.e_in / (float)W.V;
  x[3] = log2f(1.0f + (float)nsrc);
  x[4] = log2f(1.0f + (float)nent);       // entries of the level
  x[5] = log2f(1.0f + mf);                // their out-edges (push cost)
  x[6] = log2f(1.0f + fmaxf(mu, 0.0f));   // in-edges of vertices not reached by every source (pull cost)
  x[7] = x[5] - x[6];
  x[8] = log2f(1.0f + (float)d);
  x[9] = x[4] - x[0];
  x[10] = (float)pull;
  x[11] = x[10] * x[7];
  x[12] = x[10] * x[4];
}

struct GridSync {
  GridBar* bar;
  __device__ __forceinline__ bool sync() { return grid_barrier(bar); }
  __device__ __forceinline__ int tid() const { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ int nthreads() const { return gridDim.x * blockDim.x; }
};

struct BlockSync {
  __device__ __forceinline__ bool sync() {
    __syncthreads();
    return true;
  }
  __device__ __forceinline__ int tid() const { return threadIdx.x; }
  __device__ __forceinline__ int nthreads() const { return blockDim.x; }
};

// A thread-block cluster as one team: the hardware cluster barrier (release /
// acquire at cluster scope, so global-memory writes before it are seen after it).
struct ClusterSync {
  __device__ __forceinline__ bool sync() {
    cg::this_cluster().sync();
    return true;
  }
  __device__ __forceinline__ int tid() const { return (int)cg::this_cluster().thread_rank(); }
  __device__ __forceinline__ int nthreads() const { return (int)cg::this_cluster().num_threads(); }
};

__device__ __forceinline__ unsigned long long shfl64(unsigned long long x, int l) {
  unsigned lo = __shfl_sync(0xffffffffu, (unsigned)x, l);
  unsigned hi = __shfl_sync(0xffffffffu, (unsigned)(x >> 32), l);
  return ((unsigned long long)hi << 32) | lo;
}

// Entry i of a level list: a hub (more than W.hub_deg edges) when splitting is on.
// Returns true if it was queued as pieces instead of being processed here.
__device__ __forceinline__ bool queue_hub(const Work& W, int i, int lane) {
  if (W.hub_cap == 0) return false;
  const int v = W.flv[i];
  const int d = W.off[v + 1] - W.off[v];
  if (d <= W.hub_deg) return false;
  if (lane == 0) {
    const int np = (d + W.hub_chunk - 1) / W.hub_chunk;
    const unsigned long long old = atomicAdd(W.hub_cnt, (1ull << 32) | (unsigned long long)np);
    const int k = (int)(old >> 32);
    if (k < W.hub_cap) {
      W.hub_ent[k] = i;
      W.hub_base[k] = (int)(old & 0xffffffffull);
    } else {
      atomicExch(W.err, 1);
    }
  }
  return true;
}

// Piece p of the queued hubs -> (entry, edge range).
__device__ __forceinline__ void hub_piece(const Work& W, int nh, int p, int& i, int& eb, int& ee) {
  int lo = 0, hi = nh - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (W.hub_base[m] <= p) lo = m; else hi = m - 1;
  }
  i = W.hub_ent[lo];
  const int v = W.flv[i];
  eb = W.off[v] + (p - W.hub_base[lo]) * W.hub_chunk;
  ee = min(eb + W.hub_chunk, W.off[v + 1]);
}

// The next two edges with new (or successor) sources of a 32-edge chunk, for the
// half-warp form (GS = 16): lanes 0-15 take the first, lanes 16-31 the second.
__device__ __forceinline__ int half_pick(unsigned& em, int lane, int& from) {
  const int l0 = __ffs(em) - 1;
  em &= em - 1;
  int l1 = -1;
  if (em) {
    l1 = __ffs(em) - 1;
    em &= em - 1;
  }
  const int ml = lane < 16 ? l0 : l1;
  from = ml >= 0 ? ml : l0;
  return ml;
}

// GS = lanes per edge step: 32 (one lane per source bit, up to 32 * NW sources), or
// 16 when the batch has at most 16 sources, so that the two half-warps take two
// edges per step instead of leaving lanes 16-31 idle.
template <int NW, int GS>
__device__ void expand_entry(const Work& W, int i, int lane, int eb, int ee, unsigned long long* dslot = nullptr) {
  static_assert(GS == 32 || (GS == 16 && NW == 1), "half-warp steps hold up to 16 sources");
  constexpr int SW = 32 * NW;
  const int v = W.flv[i];
  const unsigned long long m = W.flm[i];
  double sv[NW];
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const int b = lane + 32 * k;
    sv[k] = ((m >> b) & 1ull) ? W.sigma[(size_t)v * SW + b] : 0.0;
  }
  const double svg = GS == 16 ? __shfl_sync(0xffffffffu, sv[0], lane & 15) : 0.0;
  // FU 32-edge chunks go together: their adj, seen and nxt accesses are each issued
  // for all chunks before any result is waited for, and their level-list appends
  // share one counter atomic.
  for (int c = eb; c < ee; c += 32 * FU) {
    int w[FU];
    unsigned long long q[FU];
    bool isnew[FU];
#pragma unroll
    for (int f = 0; f < FU; ++f) {
      const int j = c + 32 * f + lane;
      w[f] = j < ee ? W.adj[j] - W.vbase : -1;
    }
#pragma unroll
    for (int f = 0; f < FU; ++f) q[f] = w[f] >= 0 ? m & ~W.seen[w[f]] : 0ull;
#pragma unroll
    for (int f = 0; f < FU; ++f) isnew[f] = q[f] ? atomicOr(&W.nxt[w[f]], q[f]) == 0ull : false;
    unsigned nm[FU];
    int n = 0;
#pragma unroll
    for (int f = 0; f < FU; ++f) {
      nm[f] = __ballot_sync(0xffffffffu, isnew[f]);
      n += __popc(nm[f]);
    }
    if (n) {
      int base = 0;
      if (lane == 0) base = atomicAdd(W.cnt, n);
      base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
      for (int f = 0; f < FU; ++f) {
        if (isnew[f]) {
          const int pos = base + __popc(nm[f] & ((1u << lane) - 1u));
          if (pos < W.cap)
            W.flv[pos] = w[f];
          else
            atomicExch(W.err, 1);
        }
        base += __popc(nm[f]);
      }
      if (dslot) {  // the appended vertices' out-edges (the next level's push cost)
        unsigned long long ds = 0;
#pragma unroll
        for (int f = 0; f < FU; ++f)
          if (isnew[f]) ds += (unsigned long long)(W.off[w[f] + 1] - W.off[w[f]]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ds += __shfl_xor_sync(0xffffffffu, ds, o);
        if (lane == 0 && ds) atomicAdd(dslot, ds);
      }
    }
#pragma unroll
    for (int f = 0; f < FU; ++f) {
      unsigned em = __ballot_sync(0xffffffffu, q[f] != 0ull);
      while (em) {
        if (GS == 16) {
          int from;
          const int ml = half_pick(em, lane, from);
          from = max(from, 0);
          const unsigned long long qm = shfl64(q[f], from);
          const int wm = __shfl_sync(0xffffffffu, w[f], from);
          const int b = lane & 15;
          if (ml >= 0 && ((qm >> b) & 1ull)) atomicAdd(&W.sigma[(size_t)wm * SW + b], svg);
          continue;
        }
        const int l = __ffs(em) - 1;
        em &= em - 1;
        const unsigned long long ql = shfl64(q[f], l);
        const int wl = __shfl_sync(0xffffffffu, w[f], l);
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int b = lane + 32 * k;
          if ((ql >> b) & 1ull) atomicAdd(&W.sigma[(size_t)wl * SW + b], sv[k]);
        }
      }
    }
  }
}

// Pull: the parents of w among in-edges [eb, ee) that sit in the level (dense masks)
// for sources w has not reached (sw): newm gets their sources, acc[k] the sum of their
// sigma for source bit lane + 32k, in edge order. Warp-uniform newm.
template <int NW>
__device__ __forceinline__ void pull_scan(const Work& W, unsigned long long sw, int eb, int ee, int lane,
                                          unsigned long long& newm, double (&acc)[NW]) {
  constexpr int SW = 32 * NW;
  for (int c = eb; c < ee; c += 32) {
    const int j = c + lane;
    const int v = j < ee ? W.radj[j] - W.vbase : -1;
    const unsigned long long fm = v >= 0 ? W.dense[v] & ~sw : 0ull;
    unsigned em = __ballot_sync(0xffffffffu, fm != 0ull);
    while (em) {
      const int l = __ffs(em) - 1;
      em &= em - 1;
      const unsigned long long fl = shfl64(fm, l);
      const int vl = __shfl_sync(0xffffffffu, v, l);
      newm |= fl;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int b = lane + 32 * k;
        if ((fl >> b) & 1ull) acc[k] += W.sigma[(size_t)vl * SW + b];
      }
    }
  }
}

// A warp's appends to the level list, 32 at a time (one counter atomic each); the
// out-edges of the appended vertices go to ldeg[slot].
struct AppendBuf {
  int32_t* s;  // this warp's 32 slots in shared memory
  int n;       // warp-uniform
};

__device__ __forceinline__ void append_flush(const Work& W, AppendBuf& ab, int lane, int slot) {
  if (ab.n == 0) return;
  __syncwarp();
  int base = 0;
  if (lane == 0) base = atomicAdd(W.cnt, ab.n);
  base = __shfl_sync(0xffffffffu, base, 0);
  unsigned long long dsum = 0;
  if (lane < ab.n) {
    const int w = ab.s[lane];
    if (base + lane < W.cap)
      W.flv[base + lane] = w;
    else
      atomicExch(W.err, 1);
    dsum = (unsigned long long)(W.off[w + 1] - W.off[w]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
  if (lane == 0 && dsum) atomicAdd(W.ldeg + slot, dsum);
  __syncwarp();
  ab.n = 0;
}

// One pull level: the level's masks are in dense. Vertices of at most PULL_SPLIT
// in-edges are scanned by one warp each (their sigma and next mask written directly);
// the pieces of the larger ones are shared by all warps and merged with atomics (FP64
// adds of integers, exact in any order; the first piece to set a next-mask bit appends
// the vertex). `slot` = the next level's index in ldeg.
template <int NW>
__device__ void pull_level(const Work& W, unsigned long long full, int lane, int gw, int nw, int slot,
                           int32_t* s_app) {
  constexpr int SW = 32 * NW;
  AppendBuf ab{s_app + (threadIdx.x >> 5) * 32, 0};
  for (int w = gw; w < W.V; w += nw) {
    const int eb = W.roff[w], ee = W.roff[w + 1];
    if (ee - eb > PULL_SPLIT) continue;
    const unsigned long long sw = W.seen[w];
    if ((sw & full) == full || ee == eb) continue;
    unsigned long long newm = 0;
    double acc[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) acc[k] = 0.0;
    pull_scan<NW>(W, sw, eb, ee, lane, newm, acc);
    if (newm) {
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int b = lane + 32 * k;
        if ((newm >> b) & 1ull) W.sigma[(size_t)w * SW + b] = acc[k];
      }
      if (lane == 0) {
        W.nxt[w] = newm;
        ab.s[ab.n] = w;
      }
      if (++ab.n == 32) append_flush(W, ab, lane, slot);
    }
  }
  const int np = W.n_phub ? W.phub_base[W.n_phub] : 0;
  for (int p = gw; p < np; p += nw) {
    int lo = 0, hi = W.n_phub - 1;  // the last hub whose first piece <= p
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (W.phub_base[m] <= p) lo = m; else hi = m - 1;
    }
    const int w = W.phub[lo];
    const unsigned long long sw = W.seen[w];
    if ((sw & full) == full) continue;
    const int eb = W.roff[w] + (p - W.phub_base[lo]) * PULL_SPLIT;
    const int ee = min(eb + PULL_SPLIT, W.roff[w + 1]);
    unsigned long long newm = 0;
    double acc[NW];
#pragma unroll
    for (int k = 0; k < NW; ++k) acc[k] = 0.0;
    pull_scan<NW>(W, sw, eb, ee, lane, newm, acc);
    if (newm) {
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int b = lane + 32 * k;
        if ((newm >> b) & 1ull) atomicAdd(&W.sigma[(size_t)w * SW + b], acc[k]);
      }
      int first = 0;
      if (lane == 0) {
        first = atomicOr(&W.nxt[w], newm) == 0ull;
        if (first) ab.s[ab.n] = w;
      }
      first = __shfl_sync(0xffffffffu, first, 0);
      if (first && ++ab.n == 32) append_flush(W, ab, lane, slot);
    }
  }
  append_flush(W, ab, lane, slot);
}

// piece = false: the whole entry, dependencies written to delta; piece = true: an
// edge range of a hub entry, partial dependencies added to dacc (FP64 atomics).
template <int NW, int GS, int B>
__device__ void backward_entry(const Work& W, int i, int lane, int eb, int ee, bool piece) {
  static_assert(GS == 32 || (GS == 16 && NW == 1), "half-warp steps hold up to 16 sources");
  constexpr int SW = 32 * NW;
  const int v = W.flv[i];
  const unsigned long long m = W.flm[i];
  double sv[NW], acc[NW];
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const int b = lane + 32 * k;
    sv[k] = ((m >> b) & 1ull) ? W.sigma[(size_t)v * SW + b] : 0.0;
    acc[k] = 0.0;
  }
  double accg = 0.0;  // GS = 16: this half-warp's share for source bit (lane & 15)
  for (int c = eb; c < ee; c += 32) {
    const int j = c + lane;
    int w = 0;
    unsigned long long s = 0;
    if (j < ee) {
      w = W.adj[j] - W.vbase;
      s = m & W.dense[w];
    }
    // Successors are taken BU at a time: all their q loads are issued before any is
    // summed (one memory latency per BU successors instead of per successor), and the
    // sums run in edge order. q[w] = (1 + delta[w]) / sigma[w] was stored when w's
    // dependency became final, so a successor costs one 8-byte load and one add; the
    // product with sigma[v] is taken once per entry.
    unsigned em = __ballot_sync(0xffffffffu, s != 0ull);
    while (em) {
      if (GS == 16) {
        const int b = lane & 15;
        int wm[B];
        bool on[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
          int from;
          const int ml = half_pick(em, lane, from);  // -1 once em is empty
          from = max(from, 0);
          const unsigned long long sm = shfl64(s, from);
          wm[u] = __shfl_sync(0xffffffffu, w, from);
          on[u] = ml >= 0 && ((sm >> b) & 1ull);
        }
        double qs[B];
#pragma unroll
        for (int u = 0; u < B; ++u)
          if (on[u]) qs[u] = W.q[(size_t)wm[u] * SW + b];
#pragma unroll
        for (int u = 0; u < B; ++u)
          if (on[u]) accg += qs[u];
        continue;
      }
      int wl[B];
      unsigned pm = 0;  // bit u * NW + k: successor u has source bit lane + 32 k
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const bool have = em != 0u;
        const int l = have ? __ffs(em) - 1 : 0;
        em &= em - 1;
        const unsigned long long sl = shfl64(s, l);
        wl[u] = __shfl_sync(0xffffffffu, w, l);
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if (have && ((sl >> (lane + 32 * k)) & 1ull)) pm |= 1u << (u * NW + k);
      }
      double qs[B][NW];
#pragma unroll
      for (int u = 0; u < B; ++u)
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if ((pm >> (u * NW + k)) & 1u) qs[u][k] = W.q[(size_t)wl[u] * SW + lane + 32 * k];
#pragma unroll
      for (int u = 0; u < B; ++u)
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if ((pm >> (u * NW + k)) & 1u) acc[k] += qs[u][k];
    }
  }
  if (GS == 16) acc[0] = accg + __shfl_down_sync(0xffffffffu, accg, 16);  // first half, then second
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const int b = lane + 32 * k;
    if ((m >> b) & 1ull) {
      if (piece) {
        if (acc[k] != 0.0) atomicAdd(&W.dacc[(size_t)v * SW + b], acc[k]);  // partial sum of q
      } else {
        const float dv = (float)(sv[k] * acc[k]);
        W.delta[(size_t)v * SW + b] = dv;
        W.q[(size_t)v * SW + b] = (1.0 + (double)dv) / sv[k];
      }
    }
  }
}

// One batch of nsrc (<= 32*NW) sources (local ids). Every participating thread
// calls this with the same arguments; S provides the barrier and thread ranks.
// The direction of level d (every thread computes the same answer from values read
// after the same barrier): pull when the policy and the statistics say so.
__device__ __forceinline__ bool pull_this_level(const Work& W, int d, int nent, int V) {
  if (W.dir_policy == 0 || W.radj == nullptr) return false;
  if (W.dir_policy == 3) return true;
  // (policy 4, the level model, is decided in run_batch; without a model: the rule)
  if (W.dir_policy == 2) {
    unsigned h = W.dir_seed * 0x9e3779b9u ^ ((unsigned)d * 0x85ebca6bu);
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 13;
    return (h & 1u) != 0u;
  }
  // rule: a push level walks the level's out-edges with atomics on every new vertex;
  // a pull level scans the in-edges of every vertex not yet reached by all sources
  const double mf = (double)*(volatile unsigned long long*)(W.ldeg + d);
  const double mu = (double)W.e_in - (double)*(volatile unsigned long long*)W.full_in;
  return (double)W.dir_alpha * mf > mu + 0.125 * (double)V && nent > 0;
}

template <int NW, int GS, int B, class S>
__device__ bool run_batch(const Work& W, const int32_t* srcs, int nsrc, S& sync, int32_t* lvl_out = nullptr,
                          double* sig_out = nullptr, int32_t* s_app = nullptr) {
  constexpr int SW = 32 * NW;
  const int gt = sync.tid(), nt = sync.nthreads();
  const int lane = threadIdx.x & 31;
  const int gw = gt >> 5, nw = nt >> 5;
  const bool dirs = s_app != nullptr && W.dir_policy != 0 && W.radj != nullptr;
  const unsigned long long full = nsrc >= 64 ? ~0ull : ((1ull << nsrc) - 1ull);
  if (dirs) {
    for (int k = gt; k < W.maxd + 2; k += nt) W.ldeg[k] = 0ull;
    if (gt == 0) *W.full_in = 0ull;
    if (!sync.sync()) return false;
  }
  for (int k = gt; k < nsrc; k += nt) {
    const int v = srcs[k];
    W.flv[k] = v;
    W.flm[k] = 1ull << k;
    W.sigma[(size_t)v * SW + k] = 1.0;
    atomicOr(&W.seen[v], 1ull << k);
    if (dirs) atomicAdd(W.ldeg, (unsigned long long)(W.off[v + 1] - W.off[v]));
  }
  if (gt == 0) {
    W.lo[0] = 0;
    W.lo[1] = nsrc;
    *W.cnt = nsrc;
  }
  if (!sync.sync()) return false;
  int d = 0;
  while (true) {
    const int b = *(volatile int*)&W.lo[d], e = *(volatile int*)&W.lo[d + 1];
    if (b == e) break;
    if (d + 2 > W.maxd) {
      if (gt == 0) atomicExch(W.err, 2);
      return false;
    }
    bool pull;
    if (dirs && W.dir_policy == 4 && W.dmodel) {
      // the level model scores push and pull on this level's statistics; every CTA
      // evaluates the same inputs the same way, so all take the same direction
      __shared__ float s_rows[2][SP_MLP_IN];
      if (threadIdx.x < 2) level_inputs(W, d, e - b, nsrc, threadIdx.x, s_rows[threadIdx.x]);
      pull = mlp_argmin<2>(W.dmodel, s_rows) == 1;
    } else {
      pull = dirs && pull_this_level(W, d, e - b, W.V);
    }
    if (dirs && W.trace && gt == 0) {
      const int t = atomicAdd(W.tcount, 1);
      if (t < W.trace_cap) {
        float* r = W.trace + (size_t)t * LTRACE;
        level_inputs(W, d, e - b, nsrc, pull ? 1 : 0, r);
        r[SP_MLP_IN] = pull ? 1.0f : 0.0f;
        unsigned long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        W.ttime[t] = now;
      }
    }
    if (pull) {
      for (int i = b + gt; i < e; i += nt) W.dense[W.flv[i]] = W.flm[i];
      if (!sync.sync()) return false;
      pull_level<NW>(W, full, lane, gw, nw, d + 1, s_app);
      if (!sync.sync()) return false;
      for (int i = b + gt; i < e; i += nt) W.dense[W.flv[i]] = 0ull;
    } else {
      for (int i = b + gw; i < e; i += nw)
        if (!queue_hub(W, i, lane))
          expand_entry<NW, GS>(W, i, lane, W.off[W.flv[i]], W.off[W.flv[i] + 1], dirs ? W.ldeg + d + 1 : nullptr);
      if (!sync.sync()) return false;
    }
    if (!pull && W.hub_cap) {
      const unsigned long long hc = *(volatile unsigned long long*)W.hub_cnt;
      const int nh = min((int)(hc >> 32), W.hub_cap), np = (int)(hc & 0xffffffffull);
      if (nh > 0) {
        for (int p = gw; p < np; p += nw) {
          int i, eb, ee;
          hub_piece(W, nh, p, i, eb, ee);
          expand_entry<NW, GS>(W, i, lane, eb, ee, dirs ? W.ldeg + d + 1 : nullptr);
        }
        if (!sync.sync()) return false;
      }
    }
    const int c = min(*(volatile int*)W.cnt, W.cap);
    if (!pull && W.hub_cap && gt == 0) *W.hub_cnt = 0ull;  // read by every CTA before the barrier above
    for (int i = e + gt; i < c; i += nt) {
      const int w = W.flv[i];
      const unsigned long long mk = W.nxt[w];
      W.flm[i] = mk;
      const unsigned long long was = W.seen[w];
      W.seen[w] = was | mk;
      W.nxt[w] = 0ull;
      if (dirs && (was | mk) == full) atomicAdd(W.full_in, (unsigned long long)(W.roff[w + 1] - W.roff[w]));
    }
    if (gt == 0) W.lo[d + 2] = c;
    if (!sync.sync()) return false;
    ++d;
  }
  const int D = d;  // levels 0..D-1 are non-empty
  if (lvl_out) {
    // forward only: BFS level and path count of every (source, vertex), source-major
    for (int i = gt; i < W.lo[D]; i += nt) {
      const int v = W.flv[i];
      const unsigned long long mk = W.flm[i];
      int lev = 0;
      while (W.lo[lev + 1] <= i) ++lev;
      for (int k = 0; k < nsrc; ++k)
        if ((mk >> k) & 1ull) {
          lvl_out[(size_t)k * W.V + v] = lev;
          sig_out[(size_t)k * W.V + v] = W.sigma[(size_t)v * SW + k];
        }
    }
    if (!sync.sync()) return false;
  }
  for (d = (lvl_out ? 0 : D - 1); d >= 1; --d) {
    const int b1 = W.lo[d + 1], e1 = W.lo[d + 2];
    for (int i = b1 + gt; i < e1; i += nt) W.dense[W.flv[i]] = W.flm[i];
    if (!sync.sync()) return false;
    const int b0 = W.lo[d], e0 = W.lo[d + 1];
    for (int i = b0 + gw; i < e0; i += nw)
      if (!queue_hub(W, i, lane)) backward_entry<NW, GS, B>(W, i, lane, W.off[W.flv[i]], W.off[W.flv[i] + 1], false);
    if (!sync.sync()) return false;
    if (W.hub_cap) {
      const unsigned long long hc = *(volatile unsigned long long*)W.hub_cnt;
      const int nh = min((int)(hc >> 32), W.hub_cap), np = (int)(hc & 0xffffffffull);
      if (nh > 0) {
        for (int p = gw; p < np; p += nw) {
          int i, eb, ee;
          hub_piece(W, nh, p, i, eb, ee);
          backward_entry<NW, GS, B>(W, i, lane, eb, ee, true);
        }
        if (!sync.sync()) return false;
        // hub dependencies: FP64 partials -> delta, scratch back to zero
        for (int k = gw; k < nh; k += nw) {
          const int i = W.hub_ent[k];
          const int v = W.flv[i];
          const unsigned long long m = W.flm[i];
#pragma unroll
          for (int q = 0; q < NW; ++q) {
            const int bb = lane + 32 * q;
            if ((m >> bb) & 1ull) {
              const size_t x = (size_t)v * SW + bb;
              const double sg = W.sigma[x];
              const float dv = (float)(sg * W.dacc[x]);
              W.delta[x] = dv;
              W.q[x] = (1.0 + (double)dv) / sg;
              W.dacc[x] = 0.0;
            }
          }
        }
        if (!sync.sync()) return false;
      }
      if (gt == 0) *W.hub_cnt = 0ull;  // every CTA read it before the barrier above
    }
    for (int i = b1 + gt; i < e1; i += nt) W.dense[W.flv[i]] = 0ull;
    if (!sync.sync()) return false;
  }
  // accumulate in source order, then reset the batch state
  for (int v = gt; v < W.V; v += nt) {
    double s = 0;
    const size_t r = (size_t)v * SW;
    for (int k = 0; k < nsrc; ++k) {
      s += (double)W.delta[r + k];
      W.delta[r + k] = 0.0f;
      W.sigma[r + k] = 0.0;
    }
    W.bc[v] += s;
    W.seen[v] = 0ull;
  }
  // a full level list (err 1) truncated this batch: every CTA reads the flag after
  // the last barrier (nothing writes it after that), so all leave together
  if (!sync.sync()) return false;
  return *(volatile int*)W.err == 0;
}

// run_batch with the half-warp step when the batch has at most 16 sources (every
// thread of the team sees the same nsrc, so all take the same branch).
template <int NW, int B, class S>
__device__ bool run_batch_any(const Work& W, const int32_t* srcs, int nsrc, S& sync, int32_t* lvl_out = nullptr,
                              double* sig_out = nullptr, int32_t* s_app = nullptr) {
  if constexpr (NW == 1) {
    if (nsrc <= 16) return run_batch<1, 16, B>(W, srcs, nsrc, sync, lvl_out, sig_out, s_app);
  }
  return run_batch<NW, 32, B>(W, srcs, nsrc, sync, lvl_out, sig_out, s_app);
}

struct GridArgs {
  Work W;
  const int32_t* srcs;
  int nsrc;
  int batch;  // sources per batch (<= 32*NW)
  GridBar* bar;
  int32_t* lvl_out;  // forward-only mode (one batch): levels and sigma, source-major
  double* sig_out;
};

template <int NW>
__global__ void __launch_bounds__(GRID_THREADS, 4) k_bc_grid(GridArgs a) {
  __shared__ int32_t s_app[GRID_THREADS];  // pull levels: 32 append slots per warp
  GridSync gs{a.bar};
  for (int s0 = 0; s0 < a.nsrc; s0 += a.batch) {
    if (!run_batch_any<NW, BU>(a.W, a.srcs + s0, min(a.batch, a.nsrc - s0), gs, a.lvl_out, a.sig_out, s_app)) {
      if (threadIdx.x == 0 && a.bar->error) atomicCAS(a.W.err, 0, 3);
      return;
    }
  }
}

// ---- many small graphs: one CTA per graph, persistent, work queue
struct GraphsArgs {
  const int32_t* off;     // union CSR rows
  const int32_t* adj;     // union CSR neighbours (global ids)
  const int32_t* voff;    // [G+1] vertex ranges
  const int32_t* soff;    // [G+1] source ranges
  const int32_t* srcs;    // global source ids
  const int32_t* order;   // graphs, largest first
  int G;
  int* next;              // work-queue counter
  // per-CTA scratch (sized for the largest graph)
  double* sigma;
  float* delta;
  double* q;
  unsigned long long* masks;  // 3 * vmax per CTA
  int32_t* flv;
  unsigned long long* flm;
  int* lo;
  int* cnt;
  double* bc;             // [Vtot] FP64 accumulator (global ids)
  int vmax, cap, maxd;
  int* err;
};

template <int NW>
__global__ void __launch_bounds__(CTA_THREADS) k_bc_graphs(GraphsArgs a) {
  constexpr int SW = 32 * NW;
  __shared__ int s_g;
  __shared__ int32_t s_src[SW];
  BlockSync bs;
  const int slot = blockIdx.x;
  Work W;
  W.sigma = a.sigma + (size_t)slot * a.vmax * SW;
  W.delta = a.delta + (size_t)slot * a.vmax * SW;
  W.q = a.q + (size_t)slot * a.vmax * SW;
  W.seen = a.masks + (size_t)slot * a.vmax * 3;
  W.nxt = W.seen + a.vmax;
  W.dense = W.nxt + a.vmax;
  W.flv = a.flv + (size_t)slot * a.cap;
  W.flm = a.flm + (size_t)slot * a.cap;
  W.cap = a.cap;
  W.lo = a.lo + (size_t)slot * (a.maxd + 2);
  W.maxd = a.maxd;
  W.cnt = a.cnt + slot;
  W.err = a.err;
  W.off = a.off;
  W.adj = a.adj;
  W.hub_cap = 0;
  W.hub_deg = bc::HUB_DEG;
  W.hub_chunk = bc::HUB_CHUNK;
  W.hub_ent = W.hub_base = nullptr;
  W.hub_cnt = nullptr;
  W.dacc = nullptr;
  while (true) {
    if (threadIdx.x == 0) s_g = atomicAdd(a.next, 1);
    __syncthreads();
    const int k = s_g;
    __syncthreads();
    if (k >= a.G) break;
    const int g = a.order[k];
    const int vb = a.voff[g], n = a.voff[g + 1] - vb;
    W.off = a.off + vb;
    W.vbase = vb;
    W.V = n;
    W.bc = a.bc + vb;
    const int sb = a.soff[g], ns = a.soff[g + 1] - sb;
    for (int s0 = 0; s0 < ns; s0 += SW) {
      const int nb = min(SW, ns - s0);
      for (int t = threadIdx.x; t < nb; t += blockDim.x) s_src[t] = a.srcs[sb + s0 + t] - vb;
      __syncthreads();
      if (!run_batch_any<NW, BU_GRAPHS>(W, s_src, nb, bs)) return;
    }
  }
}

// The many-graphs form with a cluster of C CTAs per graph (C > 1): the work queue hands
// graphs to clusters, largest first, and each graph's batches run with cluster barriers,
// so a large graph gets C SMs' worth of warps instead of one CTA's.
template <int NW, int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(CTA_THREADS) k_bc_clusters(GraphsArgs a) {
  constexpr int SW = 32 * NW;
  __shared__ int s_g;
  __shared__ int32_t s_src[SW];
  cg::cluster_group cl = cg::this_cluster();
  ClusterSync cs;
  const int slot = blockIdx.x / C;
  const bool leader = cl.block_rank() == 0;
  Work W;
  W.sigma = a.sigma + (size_t)slot * a.vmax * SW;
  W.delta = a.delta + (size_t)slot * a.vmax * SW;
  W.q = a.q + (size_t)slot * a.vmax * SW;
  W.seen = a.masks + (size_t)slot * a.vmax * 3;
  W.nxt = W.seen + a.vmax;
  W.dense = W.nxt + a.vmax;
  W.flv = a.flv + (size_t)slot * a.cap;
  W.flm = a.flm + (size_t)slot * a.cap;
  W.cap = a.cap;
  W.lo = a.lo + (size_t)slot * (a.maxd + 2);
  W.maxd = a.maxd;
  W.cnt = a.cnt + slot;
  W.err = a.err;
  W.off = a.off;
  W.adj = a.adj;
  W.hub_cap = 0;
  W.hub_deg = HUB_DEG;
  W.hub_chunk = HUB_CHUNK;
  W.hub_ent = W.hub_base = nullptr;
  W.hub_cnt = nullptr;
  W.dacc = nullptr;
  while (true) {
    if (leader && threadIdx.x == 0) s_g = atomicAdd(a.next, 1);
    cl.sync();
    const int k = *cl.map_shared_rank(&s_g, 0);
    cl.sync();  // every CTA has read the leader's s_g before it is overwritten
    if (k >= a.G) break;
    const int g = a.order[k];
    const int vb = a.voff[g], n = a.voff[g + 1] - vb;
    W.off = a.off + vb;
    W.vbase = vb;
    W.V = n;
    W.bc = a.bc + vb;
    const int sb = a.soff[g], ns = a.soff[g + 1] - sb;
    for (int s0 = 0; s0 < ns; s0 += SW) {
      const int nb = min(SW, ns - s0);
      // every CTA keeps its own copy: run_batch reads srcs from the caller's CTA
      for (int t = threadIdx.x; t < nb; t += blockDim.x) s_src[t] = a.srcs[sb + s0 + t] - vb;
      __syncthreads();
      if (!run_batch_any<NW, BU_GRAPHS>(W, s_src, nb, cs)) return;
    }
  }
}

__global__ void k_stamp_time(unsigned long long* t) {
  unsigned long long now;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
  *t = now;
}

__global__ void k_zero(void* p, size_t words) {
  unsigned long long* q = (unsigned long long*)p;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) q[i] = 0ull;
}

__global__ void k_to_float(const double* __restrict__ a, float* __restrict__ b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// ---- plain form: the generated/manual CUDA shape (one thread per vertex per level,
// host loop on a flag; bcManualv5.cu:55-105, backend_cuda/dsl_cpp_generator.cpp:275-437)
__global__ void k_plain_init(int V, int src, int* level, double* sigma, float* delta) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) {
    level[v] = v == src ? 0 : -1;
    sigma[v] = v == src ? 1.0 : 0.0;
    delta[v] = 0.0f;
  }
}

__global__ void k_plain_fwd(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ adj, int* level,
                            double* sigma, int d, int* more) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V || level[v] != d) return;
  for (int e = off[v]; e < off[v + 1]; ++e) {
    int w = adj[e];
    int old = atomicCAS(&level[w], -1, d + 1);
    if (old == -1) *more = 1;
    if (old == -1 || old == d + 1) atomicAdd(&sigma[w], sigma[v]);
  }
}

__global__ void k_plain_bwd(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const int* level, const double* sigma, float* delta, double* bc, int d) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V || level[v] != d) return;
  double acc = 0;
  for (int e = off[v]; e < off[v + 1]; ++e) {
    int w = adj[e];
    if (level[w] == d + 1) acc += sigma[v] / sigma[w] * (1.0 + (double)delta[w]);
  }
  delta[v] = (float)acc;
  bc[v] += acc;
}

}  // namespace bc

unsigned mlp_level_model(std::vector<float>& packed);  // sp_mlp.cu

struct BcPlan {
  dbuf<float> dmodel;  // the level model on the device
  unsigned dmodel_gen = 0;
  // pull levels: the vertices of more than PULL_SPLIT in-edges and their piece prefix
  // (built once per graph), the per-level out-edge counts and the reached in-edges
  bool phub_built = false;
  int n_phub = 0;
  dbuf<int32_t> phub, phub_base;
  dbuf<unsigned long long> ldeg;
  dbuf<float> trace;
  dbuf<unsigned long long> ttime;
  dbuf<int> tcount;
  int trace_n = 0;
  dbuf<double> sigma, bc, dacc, q;
  dbuf<int32_t> hub_ent, hub_base;
  dbuf<unsigned long long> hub_cnt;
  dbuf<float> delta, fout;
  dbuf<unsigned long long> masks, flm;
  dbuf<int32_t> flv, lo, cnt, srcs, level, aux;
  dbuf<GridBar> bar;
  dbuf<int> err;
  // learned variant inputs (vstat < 0: not yet) and the choice for var_nsrc sources
  int vstat = -1;
  int64_t vmax = 0, vsq = 0, vrows[4] = {}, vedges[4] = {};
  int var_choice = -1, var_nsrc = 0;
  unsigned var_gen = 0;
};

int bc_hub_deg_default() { return bc::HUB_DEG; }
int bc_cluster_default() { return bc::CLUSTER_DEFAULT; }
int bc_hub_chunk_default() { return bc::HUB_CHUNK; }

void free_bc_plan(BcPlan* p) { delete p; }

// ---- learned kernel variant -------------------------------------------------------
// The degree above which a level-list entry is cut into pieces that all warps share, and
// the piece size. Entry 3 is the fixed default (64, 64).
namespace bc {
struct Variant {
  int hub_deg, hub_chunk;
};
constexpr int VHUB[4] = {32, 64, 256, 4096};
constexpr Variant VARIANTS[] = {{32, 64},   {32, 128},  {32, 256},  {64, 64},    {64, 128},   {64, 256},
                                {256, 64},  {256, 128}, {256, 256}, {4096, 64}, {4096, 128}, {4096, 256}};
constexpr int N_VARIANTS = (int)(sizeof(VARIANTS) / sizeof(VARIANTS[0]));
constexpr int DEFAULT_VARIANT = 3;
}  // namespace bc

int bc_variant_count() { return bc::N_VARIANTS; }

// Inputs: graph shape, symmetry, the batch's source count, the share of entries in rows
// above 4096, then the candidate: its threshold and piece size, the share of entries and
// the rows that the threshold splits.
int bc_variant_features(sp_graph* g, int cand, int nsrc, float* x, int* applicable) {
  if (cand < 0 || cand >= bc::N_VARIANTS) return SP_ERR_INVALID;
  if (!g->bc) g->bc = new BcPlan();
  BcPlan* p = g->bc;
  if (p->vstat < 0) {
    SP_TRY(ensure_symmetry(g));
    DegStats ds;
    SP_TRY(degree_stats(g->off.p, g->V, bc::VHUB, 4, g->stream, &ds));
    p->vmax = ds.max_deg;
    p->vsq = ds.sum_sq;
    for (int i = 0; i < 4; ++i) {
      p->vrows[i] = ds.rows_above[i];
      p->vedges[i] = ds.edges_above[i];
    }
    p->vstat = 1;
  }
  const bc::Variant& c = bc::VARIANTS[cand];
  int t = 0;
  while (bc::VHUB[t] != c.hub_deg) ++t;
  const double V = g->V, E = std::max<double>(1.0, (double)g->E), avg = E / std::max(1.0, V);
  x[0] = (float)std::log2(std::max(1.0, V));
  x[1] = (float)std::log2(E + 1.0);
  x[2] = (float)avg;
  x[3] = (float)std::log2((double)p->vmax + 1.0);
  x[4] = (float)std::log2((double)p->vsq / E + 1.0);
  x[5] = (float)(g->symmetric > 0);
  x[6] = (float)std::log2((double)std::max(1, nsrc));
  x[7] = (float)((double)p->vedges[3] / E);
  x[8] = (float)std::log2((double)c.hub_deg);
  x[9] = (float)std::log2((double)c.hub_chunk);
  x[10] = (float)((double)p->vedges[t] / E);
  x[11] = (float)std::log2((double)p->vrows[t] + 1.0);
  x[12] = (float)std::log2((double)c.hub_deg / c.hub_chunk);
  *applicable = 1;
  return SP_OK;
}

static int bc_variant_pick(sp_graph* g, int nsrc, int* cand) {
  *cand = -1;
  const int mode = g->variant[VAR_BC];
  if (mode >= 0) {
    *cand = mode;
    return SP_OK;
  }
  if (mode != -1 || g->bc_hub_deg > 0 || g->bc_hub_chunk > 0) return SP_OK;
  const unsigned gen = variant_generation(VAR_BC);
  if (!gen) return SP_OK;
  BcPlan* p = g->bc;
  if (p->var_gen == gen && p->var_nsrc == nsrc && p->var_choice >= 0) {
    *cand = p->var_choice;
    return SP_OK;
  }
  std::vector<float> X((size_t)bc::N_VARIANTS * SP_MLP_IN);
  std::vector<int> ok(bc::N_VARIANTS);
  for (int k = 0; k < bc::N_VARIANTS; ++k)
    SP_TRY(bc_variant_features(g, k, nsrc, X.data() + (size_t)k * SP_MLP_IN, &ok[k]));
  int best = -1;
  const int st = variant_choose(VAR_BC, X, ok, bc::DEFAULT_VARIANT, g->stream, &best);
  if (st == SP_ERR_UNSUPPORTED) return SP_OK;
  SP_TRY(st);
  p->var_choice = best;
  p->var_gen = gen;
  p->var_nsrc = nsrc;
  *cand = best;
  return SP_OK;
}

static int bc_grid(sp_graph* g, const int32_t* d_srcs, int nsrc, int batch_hint, int32_t* lvl_out = nullptr,
                   double* sig_out = nullptr) {
  BcPlan* p = g->bc;
  cudaStream_t s = g->stream;
  const int V = g->V;
  const int NW = (batch_hint > 32) ? 2 : 1;
  const int SW = 32 * NW;
  const int batch = std::max(1, std::min(batch_hint, SW));
  const int maxd = 1 << 14;
  const size_t cap = (size_t)V * std::min(batch, 16) + 1024;  // level-list entries (vertex, mask)
  SP_TRY(p->sigma.alloc((size_t)V * SW));
  SP_TRY(p->delta.alloc((size_t)V * SW));
  SP_TRY(p->q.alloc((size_t)V * SW));
  SP_TRY(p->masks.alloc((size_t)V * 3));
  SP_TRY(p->flv.alloc(cap));
  SP_TRY(p->flm.alloc(cap));
  SP_TRY(p->lo.alloc(maxd + 2));
  SP_TRY(p->cnt.alloc(1));
  SP_TRY(p->bc.alloc(V));
  SP_TRY(p->bar.alloc(1));
  SP_TRY(p->err.alloc(1));
  const int hub_cap = V;
  SP_TRY(p->hub_ent.alloc(hub_cap));
  SP_TRY(p->hub_base.alloc(hub_cap));
  SP_TRY(p->hub_cnt.alloc(1));
  SP_TRY(p->dacc.alloc((size_t)V * SW));
  SP_CHECK_CUDA(cudaMemsetAsync(p->hub_cnt.p, 0, sizeof(unsigned long long), s));
  const int zg = num_sms() * 8;
  bc::k_zero<<<zg, 256, 0, s>>>(p->dacc.p, (size_t)V * SW);
  g_launches++;
  bc::k_zero<<<zg, 256, 0, s>>>(p->sigma.p, (size_t)V * SW);
  bc::k_zero<<<zg, 256, 0, s>>>(p->delta.p, (size_t)V * SW / 2);
  bc::k_zero<<<zg, 256, 0, s>>>(p->masks.p, (size_t)V * 3);
  bc::k_zero<<<zg, 256, 0, s>>>(p->bc.p, (size_t)V);
  g_launches += 4;
  SP_CHECK_CUDA(cudaMemsetAsync(p->bar.p, 0, sizeof(GridBar), s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->err.p, 0, sizeof(int), s));
  bc::GridArgs a;
  bc::Work& W = a.W;
  W.off = g->off.p;
  W.adj = g->adj.p;
  W.vbase = 0;
  W.V = V;
  W.sigma = p->sigma.p;
  W.delta = p->delta.p;
  W.q = p->q.p;
  W.seen = p->masks.p;
  W.nxt = p->masks.p + V;
  W.dense = p->masks.p + 2 * (size_t)V;
  W.flv = p->flv.p;
  W.flm = p->flm.p;
  W.cap = (int)std::min<size_t>(cap, INT_MAX);
  W.lo = p->lo.p;
  W.maxd = maxd;
  W.cnt = p->cnt.p;
  W.bc = p->bc.p;
  W.err = p->err.p;
  W.hub_ent = p->hub_ent.p;
  W.hub_base = p->hub_base.p;
  W.hub_cnt = p->hub_cnt.p;
  W.hub_cap = hub_cap;
  W.hub_deg = g->bc_hub_deg > 0 ? g->bc_hub_deg : bc::HUB_DEG;
  W.hub_chunk = g->bc_hub_chunk > 0 ? g->bc_hub_chunk : bc::HUB_CHUNK;
  {
    int cand = -1;
    SP_TRY(bc_variant_pick(g, nsrc, &cand));
    if (cand >= 0) {
      W.hub_deg = bc::VARIANTS[cand].hub_deg;
      W.hub_chunk = bc::VARIANTS[cand].hub_chunk;
    }
    g->last_variant[VAR_BC] = cand;
  }
  W.dacc = p->dacc.p;
  // forward direction per level
  std::vector<float> packed;
  const unsigned lgen = mlp_level_model(packed);
  W.dir_policy = g->bc_dir >= 0 ? g->bc_dir : (lgen ? 4 : bc::DIR_DEFAULT);
  W.dmodel = nullptr;
  if (W.dir_policy == 4 && lgen) {
    if (p->dmodel_gen != lgen) {
      SP_TRY(p->dmodel.alloc(packed.size()));
      SP_CHECK_CUDA(cudaMemcpyAsync(p->dmodel.p, packed.data(), sizeof(float) * packed.size(),
                                    cudaMemcpyHostToDevice, s));
      p->dmodel_gen = lgen;
    }
    W.dmodel = p->dmodel.p;
  }
  W.dir_alpha = g->bc_pull_alpha > 0 ? (float)g->bc_pull_alpha / 1000.0f : bc::PULL_ALPHA;
  W.dir_seed = (unsigned)g->bc_dir_seed;
  W.roff = nullptr;
  W.radj = nullptr;
  W.phub = nullptr;
  W.phub_base = nullptr;
  W.n_phub = 0;
  W.e_in = g->E;
  W.trace = nullptr;
  W.ttime = nullptr;
  W.trace_cap = 0;
  W.tcount = nullptr;
  p->trace_n = 0;
  if (W.dir_policy != 0) {
    SP_TRY(ensure_reverse(g));
    if (!p->phub_built) {
      std::vector<int32_t> roff(V + 1);
      SP_TRY(copy_out(roff.data(), g->roff.p, sizeof(int32_t) * (V + 1), s));
      std::vector<int32_t> hubs, base{0};
      for (int v = 0; v < V; ++v) {
        const int d = roff[v + 1] - roff[v];
        if (d > bc::PULL_SPLIT) {
          hubs.push_back(v);
          base.push_back(base.back() + (d + bc::PULL_SPLIT - 1) / bc::PULL_SPLIT);
        }
      }
      p->n_phub = (int)hubs.size();
      SP_TRY(p->phub.alloc(std::max<size_t>(1, hubs.size())));
      SP_TRY(p->phub_base.alloc(base.size()));
      if (!hubs.empty())
        SP_CHECK_CUDA(cudaMemcpyAsync(p->phub.p, hubs.data(), sizeof(int32_t) * hubs.size(), cudaMemcpyHostToDevice, s));
      SP_CHECK_CUDA(cudaMemcpyAsync(p->phub_base.p, base.data(), sizeof(int32_t) * base.size(), cudaMemcpyHostToDevice, s));
      SP_CHECK_CUDA(cudaStreamSynchronize(s));
      p->phub_built = true;
    }
    SP_TRY(p->ldeg.alloc((size_t)maxd + 3));  // per level, then the reached in-edges
    W.roff = g->roff.p;
    W.radj = g->radj.p;
    W.phub = p->phub.p;
    W.phub_base = p->phub_base.p;
    W.n_phub = p->n_phub;
    W.ldeg = p->ldeg.p;
    W.full_in = p->ldeg.p + maxd + 2;
    if (g->bc_trace) {
      constexpr int CAP = 1 << 14;
      SP_TRY(p->trace.alloc((size_t)CAP * bc::LTRACE));
      SP_TRY(p->ttime.alloc((size_t)CAP + 1));
      SP_TRY(p->tcount.alloc(1));
      SP_CHECK_CUDA(cudaMemsetAsync(p->tcount.p, 0, sizeof(int), s));
      W.trace = p->trace.p;
      W.ttime = p->ttime.p;
      W.trace_cap = CAP;
      W.tcount = p->tcount.p;
    }
  }
  a.srcs = d_srcs;
  a.nsrc = nsrc;
  a.batch = batch;
  a.bar = p->bar.p;
  a.lvl_out = lvl_out;
  a.sig_out = sig_out;
  void* params[] = {&a};
  int per_sm = 0;
  const void* fn = NW == 2 ? (const void*)bc::k_bc_grid<2> : (const void*)bc::k_bc_grid<1>;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bc::GRID_THREADS, 0));
  const int grid = num_sms() * std::max(1, std::min(per_sm, 4));
  SP_CHECK_CUDA(cudaLaunchCooperativeKernel(fn, grid, bc::GRID_THREADS, params, 0, s));
  g_launches++;
  int herr = 0;
  SP_TRY(copy_out(&herr, p->err.p, sizeof(int), s));
  if (herr) {
    set_error("sp_bc: device error %d (1 level lists full, 2 deeper than %d levels, 3 barrier timeout)", herr, maxd);
    return herr == 3 ? SP_ERR_TIMEOUT : SP_ERR_UNSUPPORTED;
  }
  if (W.trace) {  // the end of the last traced level
    int n = 0;
    SP_TRY(copy_out(&n, p->tcount.p, sizeof(int), s));
    p->trace_n = std::min(n, W.trace_cap);
    bc::k_stamp_time<<<1, 1, 0, s>>>(p->ttime.p + p->trace_n);
    SP_CHECK_LAUNCH();
  }
  return SP_OK;
}

static int bc_plain(sp_graph* g, const int32_t* h_srcs, int nsrc) {
  BcPlan* p = g->bc;
  cudaStream_t s = g->stream;
  const int V = g->V;
  SP_TRY(p->level.alloc(V));
  SP_TRY(p->sigma.alloc(V));
  SP_TRY(p->delta.alloc(V));
  SP_TRY(p->bc.alloc(V));
  SP_TRY(p->aux.alloc(1));
  SP_CHECK_CUDA(cudaMemsetAsync(p->bc.p, 0, sizeof(double) * V, s));
  const int tb = 1024, nb = (V + tb - 1) / tb;  // bcManualv5.cu:198-203 launch shape
  for (int k = 0; k < nsrc; ++k) {
    bc::k_plain_init<<<nb, tb, 0, s>>>(V, h_srcs[k], p->level.p, p->sigma.p, p->delta.p);
    SP_CHECK_LAUNCH();
    int d = 0;
    while (true) {
      SP_CHECK_CUDA(cudaMemsetAsync(p->aux.p, 0, sizeof(int), s));
      bc::k_plain_fwd<<<nb, tb, 0, s>>>(V, g->off.p, g->adj.p, p->level.p, p->sigma.p, d, p->aux.p);
      SP_CHECK_LAUNCH();
      int more = 0;
      SP_TRY(copy_out(&more, p->aux.p, sizeof(int), s));
      if (!more) break;
      ++d;
    }
    for (; d >= 1; --d) {
      bc::k_plain_bwd<<<nb, tb, 0, s>>>(V, g->off.p, g->adj.p, p->level.p, p->sigma.p, p->delta.p, p->bc.p, d);
      SP_CHECK_LAUNCH();
    }
  }
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_bc(sp_graph_h g, const int32_t* sources, int32_t nsrc, float* BC, int32_t variant) {
  if (!g || !BC || (nsrc > 0 && !sources) || nsrc < 0) {
    set_error("sp_bc: invalid argument");
    return SP_ERR_INVALID;
  }
  if (!g->bc) g->bc = new BcPlan();
  BcPlan* p = g->bc;
  cudaStream_t s = g->stream;
  std::vector<int32_t> hs(nsrc);
  if (nsrc) SP_CHECK_CUDA(cudaMemcpyAsync(hs.data(), sources, sizeof(int32_t) * nsrc, cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  {
    // std::set<int> semantics: each source once; ids must be vertices
    std::vector<int32_t> u = hs;
    std::sort(u.begin(), u.end());
    if (std::adjacent_find(u.begin(), u.end()) != u.end()) {
      set_error("sp_bc: repeated source (the reference takes a std::set)");
      return SP_ERR_INVALID;
    }
    if (nsrc && (u.front() < 0 || u.back() >= g->V)) {
      set_error("sp_bc: source out of range");
      return SP_ERR_INVALID;
    }
  }
  SP_TRY(p->fout.alloc(g->V));
  if (nsrc == 0) {
    SP_CHECK_CUDA(cudaMemsetAsync(p->fout.p, 0, sizeof(float) * g->V, s));
  } else if (variant == SP_BC_PLAIN) {
    SP_TRY(bc_plain(g, hs.data(), nsrc));
    bc::k_to_float<<<num_sms() * 4, 256, 0, s>>>(p->bc.p, p->fout.p, g->V);
    SP_CHECK_LAUNCH();
  } else if (variant == SP_BC_BATCHED) {
    SP_TRY(p->srcs.alloc(nsrc));
    SP_CHECK_CUDA(cudaMemcpyAsync(p->srcs.p, hs.data(), sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
    const int batch = g->bc_batch > 0 ? (int)g->bc_batch : 64;
    int st = bc_grid(g, p->srcs.p, nsrc, batch);
    // level lists hold at most V * min(batch, 16) entries; a deep graph can need more
    // when many sources share a batch, so retry with 16 sources per batch (always fits)
    if (st == SP_ERR_UNSUPPORTED && batch > 16) st = bc_grid(g, p->srcs.p, nsrc, 16);
    SP_TRY(st);
    bc::k_to_float<<<num_sms() * 4, 256, 0, s>>>(p->bc.p, p->fout.p, g->V);
    SP_CHECK_LAUNCH();
  } else {
    set_error("sp_bc: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  return copy_out(BC, p->fout.p, sizeof(float) * g->V, s);
}

extern "C" int sp_bc_graphs(sp_graph_h g, int32_t ngraphs, const int32_t* vertex_offset, const int32_t* source_offset,
                            const int32_t* sources, float* BC) {
  if (!g || ngraphs <= 0 || !vertex_offset || !source_offset || !BC) {
    set_error("sp_bc_graphs: invalid argument");
    return SP_ERR_INVALID;
  }
  if (!g->bc) g->bc = new BcPlan();
  BcPlan* p = g->bc;
  cudaStream_t s = g->stream;
  std::vector<int32_t> voff(ngraphs + 1), soff(ngraphs + 1);
  SP_CHECK_CUDA(cudaMemcpyAsync(voff.data(), vertex_offset, sizeof(int32_t) * (ngraphs + 1), cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(soff.data(), source_offset, sizeof(int32_t) * (ngraphs + 1), cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  if (voff[0] != 0 || voff[ngraphs] != g->V || soff[0] != 0) {
    set_error("sp_bc_graphs: vertex_offset must run 0..V and source_offset start at 0");
    return SP_ERR_INVALID;
  }
  int vmax = 0, smax = 0;
  for (int k = 0; k < ngraphs; ++k) {
    if (voff[k + 1] < voff[k] || soff[k + 1] < soff[k]) {
      set_error("sp_bc_graphs: offsets must be non-decreasing");
      return SP_ERR_INVALID;
    }
    vmax = std::max(vmax, voff[k + 1] - voff[k]);
    smax = std::max(smax, soff[k + 1] - soff[k]);
  }
  const int nsrc = soff[ngraphs];
  std::vector<int32_t> hs(std::max(1, nsrc));
  if (nsrc) SP_CHECK_CUDA(cudaMemcpyAsync(hs.data(), sources, sizeof(int32_t) * nsrc, cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < ngraphs; ++k) {
    std::vector<int32_t> u(hs.begin() + soff[k], hs.begin() + soff[k + 1]);
    std::sort(u.begin(), u.end());
    if (std::adjacent_find(u.begin(), u.end()) != u.end() || (!u.empty() && (u.front() < voff[k] || u.back() >= voff[k + 1]))) {
      set_error("sp_bc_graphs: sources of graph %d repeat or fall outside its vertex range", k);
      return SP_ERR_INVALID;
    }
  }
  // graphs the CTAs take from the queue, largest first
  std::vector<int32_t> order(ngraphs);
  for (int k = 0; k < ngraphs; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (int64_t)(voff[a + 1] - voff[a]) * (soff[a + 1] - soff[a]) > (int64_t)(voff[b + 1] - voff[b]) * (soff[b + 1] - soff[b]);
  });
  const int NW = smax > 32 ? 2 : 1;
  const int SW = 32 * NW;
  const int maxd = 4096;
  const int cap = vmax * std::min(std::max(1, std::min(smax, SW)), 16) + 1024;
  int per_sm = 0;
  const void* fn = NW == 2 ? (const void*)bc::k_bc_graphs<2> : (const void*)bc::k_bc_graphs<1>;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bc::CTA_THREADS, 0));
  const int C = g->bc_cluster > 0 ? g->bc_cluster : bc::CLUSTER_DEFAULT;
  // one scratch slot per team (a CTA, or a cluster of C CTAs)
  const int teams = std::max(1, std::min(num_sms() * std::max(1, std::min(per_sm, 2)) / C, ngraphs));
  const int ctas = teams;
  SP_TRY(p->sigma.alloc((size_t)ctas * vmax * SW));
  SP_TRY(p->delta.alloc((size_t)ctas * vmax * SW));
  SP_TRY(p->q.alloc((size_t)ctas * vmax * SW));
  SP_TRY(p->masks.alloc((size_t)ctas * vmax * 3));
  SP_TRY(p->flv.alloc((size_t)ctas * cap));
  SP_TRY(p->flm.alloc((size_t)ctas * cap));
  SP_TRY(p->lo.alloc((size_t)ctas * (maxd + 2)));
  SP_TRY(p->cnt.alloc(ctas + 1));
  SP_TRY(p->bc.alloc(g->V));
  SP_TRY(p->srcs.alloc(std::max(1, nsrc) + 2 * (ngraphs + 1) + ngraphs));
  SP_TRY(p->err.alloc(1));
  SP_TRY(p->fout.alloc(g->V));
  int32_t* d_srcs = p->srcs.p;
  int32_t* d_voff = d_srcs + std::max(1, nsrc);
  int32_t* d_soff = d_voff + ngraphs + 1;
  int32_t* d_order = d_soff + ngraphs + 1;
  if (nsrc) SP_CHECK_CUDA(cudaMemcpyAsync(d_srcs, hs.data(), sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(d_voff, voff.data(), sizeof(int32_t) * (ngraphs + 1), cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(d_soff, soff.data(), sizeof(int32_t) * (ngraphs + 1), cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(d_order, order.data(), sizeof(int32_t) * ngraphs, cudaMemcpyHostToDevice, s));
  const int zg = num_sms() * 8;
  bc::k_zero<<<zg, 256, 0, s>>>(p->sigma.p, (size_t)ctas * vmax * SW);
  bc::k_zero<<<zg, 256, 0, s>>>(p->delta.p, (size_t)ctas * vmax * SW / 2);
  bc::k_zero<<<zg, 256, 0, s>>>(p->masks.p, (size_t)ctas * vmax * 3);
  bc::k_zero<<<zg, 256, 0, s>>>(p->bc.p, (size_t)g->V);
  g_launches += 4;
  SP_CHECK_CUDA(cudaMemsetAsync(p->cnt.p, 0, sizeof(int) * (ctas + 1), s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->err.p, 0, sizeof(int), s));
  bc::GraphsArgs a;
  a.off = g->off.p;
  a.adj = g->adj.p;
  a.voff = d_voff;
  a.soff = d_soff;
  a.srcs = d_srcs;
  a.order = d_order;
  a.G = ngraphs;
  a.next = p->cnt.p + ctas;
  a.sigma = p->sigma.p;
  a.delta = p->delta.p;
  a.q = p->q.p;
  a.masks = p->masks.p;
  a.flv = p->flv.p;
  a.flm = p->flm.p;
  a.lo = p->lo.p;
  a.cnt = p->cnt.p;
  a.bc = p->bc.p;
  a.vmax = vmax;
  a.cap = cap;
  a.maxd = maxd;
  a.err = p->err.p;
  if (C == 1) {
    if (NW == 2)
      bc::k_bc_graphs<2><<<teams, bc::CTA_THREADS, 0, s>>>(a);
    else
      bc::k_bc_graphs<1><<<teams, bc::CTA_THREADS, 0, s>>>(a);
  } else {
    const int grid = teams * C;
#define SP_BC_CLUSTERS(CC)                                                          \
  if (NW == 2)                                                                     \
    bc::k_bc_clusters<2, CC><<<grid, bc::CTA_THREADS, 0, s>>>(a);                  \
  else                                                                             \
    bc::k_bc_clusters<1, CC><<<grid, bc::CTA_THREADS, 0, s>>>(a);
    if (C == 2) {
      SP_BC_CLUSTERS(2)
    } else if (C == 4) {
      SP_BC_CLUSTERS(4)
    } else {
      SP_BC_CLUSTERS(8)
    }
#undef SP_BC_CLUSTERS
  }
  SP_CHECK_LAUNCH();
  int herr = 0;
  SP_TRY(copy_out(&herr, p->err.p, sizeof(int), s));
  if (herr) {
    set_error("sp_bc_graphs: device error %d (1 level lists full, 2 deeper than %d levels)", herr, maxd);
    return SP_ERR_UNSUPPORTED;
  }
  bc::k_to_float<<<num_sms() * 4, 256, 0, s>>>(p->bc.p, p->fout.p, g->V);
  SP_CHECK_LAUNCH();
  return copy_out(BC, p->fout.p, sizeof(float) * g->V, s);
}

namespace sp {
// Levels (-1 = unreached) and path counts of up to 64 distinct sources (device ids in
// d_srcs) into device buffers lvl_out / sig_out of nsrc * V entries, source-major:
// the forward pass of the batched BC kernel. A pass over more than 16 sources can fill
// its level lists (a vertex is listed once per distinct level among the sources);
// then the outputs are cleared and the sources run again 16 at a time, which always fits.
int bc_levels(sp_graph* g, const int32_t* d_srcs, int nsrc, int32_t* lvl_out, double* sig_out) {
  if (!g->bc) g->bc = new BcPlan();
  cudaStream_t s = g->stream;
  const size_t V = (size_t)g->V;
  auto clear = [&]() -> int {
    SP_CHECK_CUDA(cudaMemsetAsync(lvl_out, 0xff, sizeof(int32_t) * V * nsrc, s));
    SP_CHECK_CUDA(cudaMemsetAsync(sig_out, 0, sizeof(double) * V * nsrc, s));
    return SP_OK;
  };
  SP_TRY(clear());
  int st = bc_grid(g, d_srcs, nsrc, 64, lvl_out, sig_out);
  if (st != SP_ERR_UNSUPPORTED || nsrc <= 16) return st;
  SP_TRY(clear());
  for (int k = 0; k < nsrc; k += 16)
    SP_TRY(bc_grid(g, d_srcs + k, std::min(16, nsrc - k), 16, lvl_out + V * k, sig_out + V * k));
  return SP_OK;
}
}  // namespace sp

extern "C" int sp_bfs_sigma(sp_graph_h g, const int32_t* sources, int32_t nsrc, int32_t* level, double* sigma) {
  if (!g || !sources || nsrc <= 0 || nsrc > 64 || !level || !sigma) {
    set_error("sp_bfs_sigma: invalid argument (1..64 sources)");
    return SP_ERR_INVALID;
  }
  if (!g->bc) g->bc = new BcPlan();
  BcPlan* p = g->bc;
  cudaStream_t s = g->stream;
  std::vector<int32_t> hs(nsrc);
  SP_CHECK_CUDA(cudaMemcpyAsync(hs.data(), sources, sizeof(int32_t) * nsrc, cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> u = hs;
  std::sort(u.begin(), u.end());
  if (std::adjacent_find(u.begin(), u.end()) != u.end() || u.front() < 0 || u.back() >= g->V) {
    set_error("sp_bfs_sigma: sources must be distinct vertices");
    return SP_ERR_INVALID;
  }
  const size_t n = (size_t)nsrc * g->V;
  dbuf<int32_t> dl;
  dbuf<double> ds;
  SP_TRY(dl.alloc(n));
  SP_TRY(ds.alloc(n));
  SP_TRY(p->srcs.alloc(nsrc));
  SP_CHECK_CUDA(cudaMemcpyAsync(p->srcs.p, hs.data(), sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  SP_TRY(bc_levels(g, p->srcs.p, nsrc, dl.p, ds.p));
  SP_TRY(copy_out(level, dl.p, sizeof(int32_t) * n, s));
  return copy_out(sigma, ds.p, sizeof(double) * n, s);
}

// DynBC's Batch block (dynamicDSLCodes/dynamicDecBC:271-347, dynamicBatchIncNorm:231-290,
// dynamicBatchDecNorm:280-353): the batch, then BC over the seeds on the updated graph.
// The DSL keeps every seed's BFS levels, path counts and dependencies and repairs those
// the batch reaches; this runs the batched Brandes pass again, whose cost is one forward
// and one backward sweep per 64 seeds.
extern "C" int sp_bc_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                             const int32_t* weight, const int32_t* sources, int32_t nsrc, float* BC) {
  using namespace sp;
  if (!g || !BC || nsrc < 0 || (nsrc > 0 && !sources) || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_bc_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  std::vector<int32_t> hs(nsrc);
  if (nsrc) SP_TRY(copy_out(hs.data(), sources, sizeof(int32_t) * nsrc, g->stream));  // host or device ids
  for (int32_t v : hs)
    if (v < 0 || v >= g->V) {  // checked before the batch changes anything
      set_error("sp_bc_dynamic: source %d out of range [0, %d)", v, g->V);
      return SP_ERR_INVALID;
    }
  if (n > 0) SP_TRY(update_graph(g, n, type, src, dst, weight));
  return sp_bc(g, hs.data(), nsrc, BC, SP_BC_BATCHED);
}

extern "C" int sp_bc_level_trace(sp_graph_h g, float* records, unsigned long long* times, int32_t cap, int32_t* n) {
  using namespace sp;
  if (!g || !n || cap < 0 || (cap > 0 && (!records || !times))) {
    set_error("sp_bc_level_trace: invalid argument");
    return SP_ERR_INVALID;
  }
  const int have = g->bc ? g->bc->trace_n : 0;
  *n = have;
  const int k = std::min(have, (int)cap);
  if (k == 0) return SP_OK;
  SP_TRY(copy_out(records, g->bc->trace.p, sizeof(float) * bc::LTRACE * k, g->stream));
  return copy_out(times, g->bc->ttime.p, sizeof(unsigned long long) * (k + 1), g->stream);
}
