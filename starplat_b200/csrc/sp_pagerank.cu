// PageRank, pull form over the reverse CSR, for sm_100a.
//
// Semantics: DSL staticDSLCodes/PageRankDSLV3:1-25 as emitted by the CUDA generator
// (backend_cuda/dsl_cpp_generator.cpp:1472-1480 reads d_src = srcList, count_outNbrs
// :3113-3121): pr0 = 1/V; pr'[v] = (1-delta)/V + delta * sum_{u->v} pr[u]/outdeg(u);
// diff = sum |pr' - pr|; repeat while diff > beta && iter < maxIter.
//
// Design (all iterations captured in one CUDA graph, no host round trip):
//  * Every iteration writes contrib[v] = pr[v]/outdeg(v) next to pr[v], so the next
//    gather reads one float per in-edge (the per-edge quotient the reference forms).
//  * Vertices are relabelled by out-degree (descending) once per graph and each
//    row's in-neighbours are sorted by the new ids, so the sources gathered most
//    often share cache lines and form a prefix of every row.
//  * Optionally (knob "pr.hot", off by default: measured slower on R-MAT 22) each
//    iteration runs in two launches split by source id: a HOT phase gathering only
//    from the first `hot` ids (a block of contrib small enough to stay in L1,
//    srcList streamed past L1) and a COLD phase gathering the rest and finalising
//    rows; a row's hot partial sum passes between the phases in FP64.
//  * Load balance by static bins built once per graph, per phase: 1, 4, 8 or 32
//    lanes per row segment (<= 4, <= 16, <= 32, <= 2048 edges) with all of a
//    segment's loads in flight at once; rows above 2048 in-edges are cut into
//    2048-edge chunks (one CTA each) and the CTA that adds a row's last chunk sums
//    the chunk partials in chunk order and finalises the row.
//  * Rows without in-edges hold (1-delta)/V from iteration 1 on: they are written in
//    iterations 0 and 1 only, and their diff term (identical for all of them) is
//    added as one exact sum of equal values.
//  * Row sums are FP64 and rounded once to FP32, every sum in a fixed order; the L1
//    diff is reduced per CTA and summed in CTA order by the last CTA of the cold
//    phase, which advances the iteration count and raises the done flag that makes
//    the graph's remaining launches return at once.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "sp_internal.cuh"

namespace sp {

namespace pr {
constexpr int THREADS = 256;
constexpr int CIPT = 8;                 // loads in flight per thread in chunk sums
constexpr int CHUNK = THREADS * CIPT;   // edges per long-row chunk (one round per CTA)
constexpr int LONG_DEG = 2048;          // rows with more in-edges are processed as chunks
constexpr int HOT_DEFAULT = 0;          // one phase: measured fastest on R-MAT 22 (12.0 vs 13.0-13.5 ms)
constexpr int HOT_MAX = 1 << 22;
constexpr int SRC_HINT_DEFAULT = 2;     // srcList loads: 0 __ldg, 1 L1::no_allocate, 2 L1::evict_first
constexpr int ORDER_DEFAULT = 0;        // vertex order: 0 out-degree, 1 in-degree class then out-degree
// Gathers from sources beyond the first L1_HOT_DEFAULT ids (the most-gathered, after
// relabelling by out-degree) bypass L1. R-MAT 22: 11.83 ms per run with every gather
// allocating, 11.65 with 32768 or 65536, 11.78 with 131072, 12.17 with 16384, 13.31 with 8192.
constexpr int L1_HOT_DEFAULT = 32768;
// srcList read 4 bytes per lane per load: 16-byte loads (pr.vec = 1) measured 0.7-3.7%
// slower on R-MAT 22 at every l1_hot setting.
constexpr int VEC_DEFAULT = 0;
// degree-bin upper bounds for 1, 4, 8 and 32 lanes per row segment
constexpr int BIN_T1 = 4, BIN_T4 = 16, BIN_T8 = 32;

struct State {
  int iter;
  int done;
  unsigned int ticket;
  int pad;
  double diff;
  double extra;  // diff terms of rows without in-edges (added by the last CTA)
};

// Row classes of one phase: bins 0-3 (32, 8, 4, 1 lanes per row segment), 4 = no
// segment in this phase, 5 = long row (chunks), 6 = no in-edges. Phase 0 puts long
// and empty rows in class 4.
constexpr int N_CLASS = 7;
constexpr int BIN_W[4] = {32, 8, 4, 1};

// A phase's warp tasks are implicit: bin k holds rows[row_base[k], row_base[k+1]) and
// task t of bin k covers 32 / W_k consecutive rows from row_base[k] + (t - task_base[k]) * (32 / W_k).
struct Phase {
  const int32_t* __restrict__ rows;   // row ids grouped by class, ascending within a class
  const int4* __restrict__ chunks;    // {row, e_begin, e_end, slot}
  const int32_t* __restrict__ chunk_long;  // long-row index of each chunk
  int row_base[5];
  int task_base[5];                   // task_base[4] = number of warp tasks
  int n_chunks;
};
}  // namespace pr

struct PrPlan {
  Arena graph_mem;        // per graph: relabelled CSR and iteration buffers
  Arena bin_mem;          // per hot setting: row classes and long-row chunks
  dspan<int32_t> new_id;  // vertex -> rank by out-degree (descending, stable)
  dspan<int32_t> od;      // out-degree, in relabelled order
  dspan<int32_t> roffp, radjp;  // reverse CSR in relabelled ids, rows sorted
  dspan<int32_t> hot_end; // per row: first edge whose source id >= hot
  dspan<float> outbuf;    // result in original vertex order
  dspan<int32_t> rows[2], chunk_long[2];
  dspan<int4> chunks[2];
  int row_base[2][5] = {}, task_base[2][5] = {};
  int n_chunks[2] = {0, 0}, n_zero = 0, n_long = 0;
  const int32_t* zrows = nullptr;  // rows without in-edges (class 6 of rows[1])
  dspan<int2> longs;      // [n_long] {first slot, slot count}
  dspan<unsigned int> long_ctr;
  dspan<double> chunk_part, part;
  dspan<double> diff_part;
  dspan<float> prb[2], con[2];
  dspan<pr::State> state;
  int hot = -1;           // hot id count the plan was built for
  int order = 0;          // vertex order (k_deg_keys)
  int nparts = 1, part_idx = 0;  // split plan: part part_idx of nparts (lay())
  int S = 0, Vp = 0;      // ids per part and the id space (nparts * S; V when not split)
  int lo = 0, hi = 0;     // this part's rows
  float pbeta = 0, pdelta = 0;  // split run: stop test and damping of sp_pagerank_part_begin
  int pmax_iter = 0;
  float* pcon[2] = {nullptr, nullptr};  // split run: the caller's all-gathered contrib buffers
  double* pdiff = nullptr;              // split run: the caller's diff (this part's, then the sum)
  bool two_phase() const { return task_base[0][4] > 0 || n_chunks[0] > 0; }
  cudaGraphExec_t exec = nullptr;
  int exec_iters = 0;
  float exec_beta = -1, exec_delta = -1;
  int exec_sh = -1;       // srcList policy, vector loads and L1 hot count the graph was captured with
  // the settings of the last call that launched its iterations directly: the graph is
  // captured only when a call repeats them, so a handle used once pays no capture
  int pend_iters = 0, pend_sh = -1;
  float pend_beta = -1, pend_delta = -1;
  // The iterations are captured on this private stream and launched on the graph's
  // stream, which may be the legacy default stream (where capture is not allowed).
  cudaStream_t cap = nullptr;
  // learned variant inputs: the share of in-edges whose source is among the 8192 / 32768
  // / 131072 highest out-degree sources, and in-degree statistics (vorder = -1: not yet)
  int vorder = -1;
  double vshare[3] = {0, 0, 0};
  int64_t vin_max = 0, vin_sq = 0;
  int var_choice = -1;     // the learned candidate for this plan, under model var_gen
  unsigned var_gen = 0;
};

int pr_order_default() { return pr::ORDER_DEFAULT; }
int pr_src_hint_default() { return pr::SRC_HINT_DEFAULT; }
int pr_l1_hot_default() { return pr::L1_HOT_DEFAULT; }
int pr_vec_default() { return pr::VEC_DEFAULT; }

void free_pr_plan(PrPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->cap) cudaStreamDestroy(p->cap);
  delete p;
}

namespace pr {

struct IterArgs {
  const int32_t* __restrict__ roff;
  const int32_t* __restrict__ radj;
  const int32_t* __restrict__ hot_end;
  const int32_t* __restrict__ od;    // out-degree per (relabelled) row
  const int2* __restrict__ longs;
  unsigned int* long_ctr;
  double* chunk_part;
  double* part;                      // hot-phase partial sums (FP64)
  double* diff_part;                 // [2 * grid] per-CTA diff partials of both phases
  State* st;
  int two_phase;                     // phase 0 runs; else only diff_part[grid, 2*grid) is written
  Phase ph[2];
  float base;   // (1 - delta) / V, in float as the DSL computes it
  float delta;
  double beta;
  int max_iter;
  int l1_hot;   // GH = 1: relabelled source ids below this allocate in L1
  double* diff_out;  // split plan: this part's L1 diff of the iteration (summed over parts by the caller)
};

__device__ __forceinline__ double finalize_row(const IterArgs& a, int r, double sum,
                                               const float* __restrict__ pr_old, float* __restrict__ pr_new,
                                               float* __restrict__ con_new) {
  const float s = (float)sum;
  const float np = __fadd_rn(a.base, __fmul_rn(a.delta, s));
  const float po = pr_old[r];
  pr_new[r] = np;
  const int od = a.od[r];
  con_new[r] = od > 0 ? __fdiv_rn(np, (float)od) : 0.0f;
  return fabs((double)np - (double)po);
}

// srcList is read once per iteration. SH picks how its loads treat L1: 0 cached
// (__ldg), 1 not allocated in L1, 2 allocated but evicted first, so that streaming it
// does not push out the contrib lines that the gathers reuse. R-MAT 22: 11.72 ms per
// run with 0, 11.68 with 1, 11.57 with 2 (contrib gathers marked evict-last on top:
// 12.0). The hot phase (PH 0) always keeps it out of L1.
template <int PH, int SH>
__device__ __forceinline__ int ld_src(const int32_t* p) {
  int v;
  if (PH == 0 || SH == 1) {
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
  }
  if (SH == 2) {
    asm("ld.global.nc.L1::evict_first.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
  }
  return __ldg(p);
}

// srcList entries i .. i+3 in one 16-byte load (i a multiple of 4; the reverse rows
// are 256-byte aligned and padded by 16 bytes, so a load that starts before E stays
// inside the buffer), with the L1 policy of ld_src.
template <int PH, int SH>
__device__ __forceinline__ int4 ld_src4(const int32_t* p) {
  int4 v;
  if (PH == 0 || SH == 1) {
    asm("ld.global.nc.L1::no_allocate.v4.b32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  } else if (SH == 2) {
    asm("ld.global.nc.L1::evict_first.v4.b32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  } else {
    v = __ldg(reinterpret_cast<const int4*>(p));
  }
  return v;
}

__device__ __forceinline__ int comp4(const int4& q, int j) { return j == 0 ? q.x : j == 1 ? q.y : j == 2 ? q.z : q.w; }

// Where a gather of contrib[u] reads from. Only global memory (through L1) is used:
// staging the hottest sources in shared memory measured 20-180% slower on R-MAT 22
// (the carve-out shrinks L1, where those sources already hit, and large tables halve
// the resident CTAs). With GH = 1 only the `hot` most-gathered sources (the lowest
// relabelled ids) are allocated in L1; a gather from any other source bypasses it, so
// the stream of cold sectors does not evict the hot lines.
template <int SH, int GH>
struct GatherGlobal {
  static constexpr int kSrcHint = SH;
  const float* __restrict__ con;
  int hot;
  __device__ __forceinline__ float operator()(int u) const {
    if (GH == 1 && u >= hot) {
      float v;
      asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(con + u));
      return v;
    }
    return __ldg(con + u);
  }
};
// Sum of con[radj[i]] for i in [b, e) by a group of W lanes (sl = lane within the
// group), U loads in flight per lane per round, reduced with a fixed xor tree.
template <int PH, int W, int U, class G>
__device__ __forceinline__ double group_row_sum(int b, int e, int sl, const int32_t* __restrict__ radj,
                                                const G& gather) {
  double acc = 0;
  for (int base = b; base < e; base += W * U) {
    int idx[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int i = base + sl + W * k;
      idx[k] = i < e ? ld_src<PH, G::kSrcHint>(radj + i) : -1;
    }
    float v[U];
#pragma unroll
    for (int k = 0; k < U; ++k) v[k] = idx[k] >= 0 ? gather(idx[k]) : 0.0f;
#pragma unroll
    for (int k = 0; k < U; ++k) acc += (double)v[k];
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// Sum of con[radj[i]] for i in [b, e) by a whole warp with 16-byte srcList loads: each
// lane loads U4 groups of four consecutive entries per round from the 4-aligned start
// below b (entries outside [b, e) are read but not gathered), then gathers all of them
// before any sum; reduced with a fixed xor tree.
template <int PH, int U4, class G>
__device__ __forceinline__ double warp_row_sum_vec(int b, int e, int lane, const int32_t* __restrict__ radj,
                                                   const G& gather) {
  double acc = 0;
  for (int base = b & ~3; base < e; base += 32 * 4 * U4) {
    int4 q[U4];
#pragma unroll
    for (int k = 0; k < U4; ++k) {
      const int i = base + 4 * lane + 128 * k;
      q[k] = i < e ? ld_src4<PH, G::kSrcHint>(radj + i) : make_int4(0, 0, 0, 0);
    }
    float v[4 * U4];
#pragma unroll
    for (int k = 0; k < U4; ++k) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = base + 4 * lane + 128 * k + j;
        v[4 * k + j] = (i >= b && i < e) ? gather(comp4(q[k], j)) : 0.0f;
      }
    }
#pragma unroll
    for (int k = 0; k < 4 * U4; ++k) acc += (double)v[k];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// One warp task: up to 32/W rows of one bin, W lanes per row segment (VEC: the 32-lane
// bin reads srcList 16 bytes at a time).
template <int PH, int W, int U, int VEC, class G>
__device__ __forceinline__ double warp_task(const IterArgs& a, int start, int count, int lane,
                                            const float* __restrict__ pr_old, const G& gather,
                                            float* __restrict__ pr_new, float* __restrict__ con_new) {
  const int g = lane / W, sl = lane % W;
  int r = -1, b = 0, e = 0, other = 0;
  if (g < count) {
    r = a.ph[PH].rows[start + g];
    const int r0 = a.roff[r], h = a.hot_end[r], r1 = a.roff[r + 1];
    if (PH == 0) {
      b = r0, e = h, other = r1 - h;  // other > 0: the row also has cold edges
    } else {
      b = h, e = r1, other = h - r0;  // other > 0: a hot partial is waiting
    }
  }
  double sum;
  if constexpr (VEC == 1 && W == 32)
    sum = warp_row_sum_vec<PH, U / 4>(b, e, lane, a.radj, gather);
  else
    sum = group_row_sum<PH, W, U>(b, e, sl, a.radj, gather);
  if (r < 0 || sl != 0) return 0.0;
  if (PH == 0) {
    if (other > 0) {
      a.part[r] = sum;
      return 0.0;
    }
    return finalize_row(a, r, sum, pr_old, pr_new, con_new);
  }
  if (other > 0) sum += a.part[r];
  return finalize_row(a, r, sum, pr_old, pr_new, con_new);
}

// One phase of one iteration by persistent CTAs of NT threads: long-row chunks
// first (a CTA each, CHUNK / NT loads per thread), then the warp tasks, heaviest
// bins first; then the diff partials (the last CTA of the cold phase sums them).
template <int PH, int NT, int VEC, class G>
__device__ __forceinline__ void phase_body(const IterArgs& a, const G& gather, const float* __restrict__ pr_old,
                                           float* __restrict__ pr_new, float* __restrict__ con_new, double* s_red,
                                           int& s_last) {
  constexpr int CI = CHUNK / NT;
  static_assert(CI * NT == CHUNK, "chunk must be a multiple of the CTA size");
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const Phase& P = a.ph[PH];
  double my_diff = 0;

  for (int ci = blockIdx.x; ci < P.n_chunks; ci += gridDim.x) {
    const int4 c = P.chunks[ci];
    double acc = 0;
    if constexpr (VEC == 1) {
      // 16-byte srcList loads from the 4-aligned start below the chunk: a second round
      // picks up the (at most three) entries past one aligned CHUNK
      constexpr int C4 = CI / 4;
      for (int base = c.y & ~3; base < c.z; base += 4 * NT * C4) {
        int4 q[C4];
#pragma unroll
        for (int k = 0; k < C4; ++k) {
          const int e = base + 4 * tid + 4 * NT * k;
          q[k] = e < c.z ? ld_src4<PH, G::kSrcHint>(a.radj + e) : make_int4(0, 0, 0, 0);
        }
        float v[CI];
#pragma unroll
        for (int k = 0; k < C4; ++k) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int e = base + 4 * tid + 4 * NT * k + j;
            v[4 * k + j] = (e >= c.y && e < c.z) ? gather(comp4(q[k], j)) : 0.0f;
          }
        }
#pragma unroll
        for (int k = 0; k < CI; ++k) acc += (double)v[k];
      }
    } else {
      int idx[CI];
#pragma unroll
      for (int k = 0; k < CI; ++k) {
        const int e = c.y + tid + k * NT;
        idx[k] = e < c.z ? ld_src<PH, G::kSrcHint>(a.radj + e) : -1;
      }
      float v[CI];
#pragma unroll
      for (int k = 0; k < CI; ++k) v[k] = idx[k] >= 0 ? gather(idx[k]) : 0.0f;
#pragma unroll
      for (int k = 0; k < CI; ++k) acc += (double)v[k];
    }
    const double tot = block_sum<NT>(acc, s_red);
    if (tid == 0) {
      a.chunk_part[c.w] = tot;
      __threadfence();
      const int li = P.chunk_long[ci];
      const int2 L = a.longs[li];
      const unsigned int old = atomicAdd(&a.long_ctr[li], 1u);
      s_last = (old == (unsigned)(L.y - 1)) ? li + 1 : 0;
    }
    __syncthreads();
    if (s_last && tid == 0) {
      __threadfence();
      const int li = s_last - 1;
      const int2 L = a.longs[li];
      double sum = 0;
      const volatile double* cp = a.chunk_part;
      for (int k = 0; k < L.y; ++k) sum += cp[L.x + k];
      my_diff += finalize_row(a, c.x, sum, pr_old, pr_new, con_new);
      a.long_ctr[li] = 0;
    }
    __syncthreads();
  }

  const int warps_total = gridDim.x * (NT / 32);
  for (int t = blockIdx.x * (NT / 32) + (tid >> 5); t < P.task_base[4]; t += warps_total) {
    const int k = (t >= P.task_base[1]) + (t >= P.task_base[2]) + (t >= P.task_base[3]);
    const int per = 32 >> (k == 0 ? 5 : k == 1 ? 3 : k == 2 ? 2 : 0);  // rows per task: 32 / W
    const int start = P.row_base[k] + (t - P.task_base[k]) * per;
    const int count = min(per, P.row_base[k + 1] - start);
    switch (k) {
      case 0: my_diff += warp_task<PH, 32, 8, VEC>(a, start, count, lane, pr_old, gather, pr_new, con_new); break;
      case 1: my_diff += warp_task<PH, 8, 4, VEC>(a, start, count, lane, pr_old, gather, pr_new, con_new); break;
      case 2: my_diff += warp_task<PH, 4, 4, VEC>(a, start, count, lane, pr_old, gather, pr_new, con_new); break;
      default: my_diff += warp_task<PH, 1, 4, VEC>(a, start, count, lane, pr_old, gather, pr_new, con_new); break;
    }
  }

  const double bd = block_sum<NT>(my_diff, s_red);
  if (PH == 0) {
    if (tid == 0) a.diff_part[blockIdx.x] = bd;
    return;
  }
  // cold phase: the last CTA sums both phases' partials in CTA order
  if (tid == 0) {
    a.diff_part[gridDim.x + blockIdx.x] = bd;
    __threadfence();
    const unsigned int t = atomicAdd(&a.st->ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const volatile double* dp = a.diff_part;
    double p = 0;
    for (int i = (a.two_phase ? 0 : (int)gridDim.x) + tid; i < 2 * (int)gridDim.x; i += NT) p += dp[i];
    const double total = block_sum<NT>(p, s_red);
    if (tid == 0) {
      const double all = total + *(volatile double*)&a.st->extra;
      if (a.diff_out) *a.diff_out = all;
      const int it = a.st->iter + 1;
      a.st->iter = it;
      a.st->diff = all;
      a.st->done = (all > a.beta && it < a.max_iter) ? 0 : 1;
      a.st->ticket = 0;
      a.st->extra = 0.0;
    }
  }
}

// One phase of one iteration, every gather from global memory (256-thread CTAs).
// SH: L1 policy of srcList loads; GH: 1 = only sources below a.l1_hot allocate in L1;
// VEC: 16-byte srcList loads in the 32-lane bin and the long-row chunks.
template <int PH, int SH, int GH, int VEC>
__global__ void __launch_bounds__(THREADS, 8) k_phase(IterArgs a, const float* __restrict__ pr_old,
                                                   const float* __restrict__ con_old, float* __restrict__ pr_new,
                                                   float* __restrict__ con_new) {
  __shared__ double s_red[THREADS / 32];
  __shared__ int s_last;
  if (a.st->done) return;
  phase_body<PH, THREADS, VEC>(a, GatherGlobal<SH, GH>{con_old, a.l1_hot}, pr_old, pr_new, con_new, s_red, s_last);
}

// Rows without in-edges, iterations 0 and 1 only: pr' = (1-delta)/V. Their diff
// terms are all |base - pr_old| (one value per iteration), so the sum is an exact
// multiple of it whatever the order of the FP64 additions.
__global__ void k_zero_rows(IterArgs a, const int32_t* __restrict__ zrows, int nz, const float* __restrict__ pr_old,
                            float* __restrict__ pr_new, float* __restrict__ con_new) {
  if (a.st->done) return;
  double d = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nz; i += gridDim.x * blockDim.x) {
    const int r = zrows[i];
    const float np = a.base;
    d += fabs((double)np - (double)pr_old[r]);
    pr_new[r] = np;
    const int od = a.od[r];
    con_new[r] = od > 0 ? __fdiv_rn(np, (float)od) : 0.0f;
  }
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0 && d != 0.0) atomicAdd(&a.st->extra, d);
}

// ---- relabelling by out-degree (descending)
// Relabelling sort keys. Order 0: out-degree, descending. Order 1: in-degree class
// first (rows of more than LONG_DEG in-edges, then the 32-, 8-, 4- and 1-lane bins,
// then rows without in-edges), out-degree descending within a class, so that each
// bin of the single-phase iteration is one contiguous id range.
__device__ __forceinline__ int indeg_class(int d) {
  return d > LONG_DEG ? 0 : d > BIN_T8 ? 1 : d > BIN_T4 ? 2 : d > BIN_T1 ? 3 : d > 0 ? 4 : 5;
}

__global__ void k_deg_keys(int V, int order, const int32_t* __restrict__ off, const int32_t* __restrict__ roff,
                           int32_t* __restrict__ key, int32_t* __restrict__ id) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int od = off[v + 1] - off[v];
    key[v] = order == 0 ? -od : (indeg_class(roff[v + 1] - roff[v]) << 28) | (0x0fffffff - min(od, 0x0fffffff));
    id[v] = v;
  }
}

// Vertex ids of a plan split into np parts (sp_pagerank_part_*): out-degree rank k goes
// to part k % np at position k / np, and part r's vertices are the id range
// [r * S, r * S + count_r). Every part's slice of contrib is then one contiguous block
// of S floats (what an all-gather of equal blocks needs), and the ranks' heavy
// vertices are dealt round-robin, so the parts' in-edge counts stay close. np = 1 is
// the identity.
__device__ __forceinline__ int lay(int k, int np, int S) { return np == 1 ? k : (k % np) * S + k / np; }

__global__ void k_relabel_rows(int V, int np, int S, const int32_t* __restrict__ inv, const int32_t* __restrict__ off,
                               int32_t* __restrict__ new_id, int32_t* __restrict__ od) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V; k += gridDim.x * blockDim.x) {
    const int v = inv[k];
    new_id[v] = lay(k, np, S);
    od[k] = off[v + 1] - off[v];
  }
}

// Out-degrees moved from rank order to the plan's ids (pads of a split plan keep 0).
__global__ void k_od_layout(int V, int np, int S, const int32_t* __restrict__ odk, int32_t* __restrict__ od) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V; k += gridDim.x * blockDim.x) od[lay(k, np, S)] = odk[k];
}

// Stable transpose, step 1: the (new dst, new src) pair of every edge, written in
// ascending new source order (source k is old vertex inv[k]; its pairs start at
// offp[k]). A warp takes 32 consecutive sources and flattens their edges over its
// lanes (an exclusive scan of the out-degrees), 32 edges per step and four steps'
// loads in flight together, so short rows do not leave lanes idle. Sources of more than 1024 out-edges are listed for
// k_fwd_pairs_big instead.
__global__ void k_fwd_pairs(int V, int np, int S, const int32_t* __restrict__ inv, const int32_t* __restrict__ new_id,
                            const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const int32_t* __restrict__ offp, const int32_t* __restrict__ od,
                            int32_t* __restrict__ dst, int32_t* __restrict__ src, int32_t* __restrict__ big,
                            int* __restrict__ nbig) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  for (int k0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; k0 < V; k0 += ((gridDim.x * blockDim.x) >> 5) * 32) {
    const int k = k0 + lane;
    int n = 0, b = 0, d = 0;
    if (k < V) {
      n = od[k];
      if (n > 1024) {
        big[atomicAdd(nbig, 1)] = k;
        n = 0;
      } else if (n > 0) {
        b = off[inv[k]];
        d = offp[k];
      }
    }
    int inc = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += t;
    }
    const int total = __shfl_sync(FULL, inc, 31);
    const int excl = inc - n;
    constexpr int U = 4;  // steps whose loads are in flight together
    for (int t0 = 0; t0 < total; t0 += 32 * U) {
      int pos[U], nb[U], row[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int t = t0 + 32 * u + lane;
        int j = 0;  // the last lane whose edges start at or before t (never a lane without edges)
#pragma unroll
        for (int s = 16; s > 0; s >>= 1)
          if (__shfl_sync(FULL, excl, j + s) <= t) j += s;
        const int jb = __shfl_sync(FULL, b, j), jd = __shfl_sync(FULL, d, j), je = __shfl_sync(FULL, excl, j);
        pos[u] = t < total ? jd + (t - je) : -1;
        nb[u] = t < total ? adj[jb + (t - je)] : 0;
        row[u] = lay(k0 + j, np, S);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) nb[u] = pos[u] >= 0 ? new_id[nb[u]] : 0;
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (pos[u] >= 0) {
          dst[pos[u]] = nb[u];
          src[pos[u]] = row[u];
        }
    }
  }
}

// Rows of more than 1024 out-edges: a CTA per row, four edges per thread in flight.
__global__ void k_fwd_pairs_big(int np, int S, const int32_t* __restrict__ inv, const int32_t* __restrict__ new_id,
                                const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                const int32_t* __restrict__ offp, const int32_t* __restrict__ od,
                                int32_t* __restrict__ dst, int32_t* __restrict__ src,
                                const int32_t* __restrict__ big, const int* __restrict__ nbig) {
  constexpr int U = 4;
  for (int i = blockIdx.x; i < *nbig; i += gridDim.x) {
    const int k = big[i];
    const int n = od[k], b = off[inv[k]], d = offp[k];
    for (int j0 = threadIdx.x; j0 < n; j0 += blockDim.x * U) {
      int a[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = j0 + u * blockDim.x;
        a[u] = j < n ? adj[b + j] : 0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = j0 + u * blockDim.x;
        if (j < n) {
          dst[d + j] = new_id[a[u]];
          src[d + j] = lay(k, np, S);
        }
      }
    }
  }
}

__device__ __forceinline__ int bin_of(int d) { return d > BIN_T8 ? 0 : d > BIN_T4 ? 1 : d > BIN_T1 ? 2 : 3; }

// Row class per phase (see N_CLASS) and the class sizes; iota[r] = r is the value
// array of the stable sort that groups rows by class.
// Rows outside [lo, hi) (another part's, or a split plan's pads) get class 4 in both
// phases: no work.
__global__ void k_row_classes(int V, int lo, int hi, const int32_t* __restrict__ roffp,
                              const int32_t* __restrict__ hot_end, uint8_t* __restrict__ key0,
                              uint8_t* __restrict__ key1, int32_t* __restrict__ iota,
                              int* __restrict__ counts /* [2 * N_CLASS] */) {
  int c0[N_CLASS], c1[N_CLASS];
#pragma unroll
  for (int j = 0; j < N_CLASS; ++j) c0[j] = c1[j] = 0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x) {
    const int b = roffp[r], e = roffp[r + 1], h = hot_end[r];
    int k0 = 4, k1;
    if (r < lo || r >= hi) {
      k1 = 4;
    } else if (e == b) {
      k1 = 6;
    } else if (e - b > LONG_DEG) {
      k1 = 5;
    } else {
      k0 = h > b ? bin_of(h - b) : 4;
      k1 = e > h ? bin_of(e - h) : 4;
    }
    key0[r] = (uint8_t)k0;
    key1[r] = (uint8_t)k1;
    iota[r] = r;
#pragma unroll
    for (int j = 0; j < N_CLASS; ++j) {
      c0[j] += k0 == j;
      c1[j] += k1 == j;
    }
  }
#pragma unroll
  for (int j = 0; j < N_CLASS; ++j) {
    const int a = __reduce_add_sync(0xffffffffu, c0[j]), b = __reduce_add_sync(0xffffffffu, c1[j]);
    if ((threadIdx.x & 31) == 0) {
      if (a) atomicAdd(&counts[j], a);
      if (b) atomicAdd(&counts[N_CLASS + j], b);
    }
  }
}

// Chunk counts of each long row's two segments packed as n0 | n1 << 32, so that one
// exclusive scan gives both phases' chunk offsets (and their sum, the row's first
// slot). Entry n_long is 0: its prefix is the total.
__global__ void k_long_counts(int n_long, const int32_t* __restrict__ lrows, const int32_t* __restrict__ roffp,
                              const int32_t* __restrict__ hot_end, unsigned long long* __restrict__ packed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_long; i += gridDim.x * blockDim.x) {
    unsigned long long v = 0;
    if (i < n_long) {
      const int r = lrows[i];
      const int b = roffp[r], h = hot_end[r], e = roffp[r + 1];
      const unsigned long long n0 = (unsigned)(h - b + CHUNK - 1) / CHUNK;
      const unsigned long long n1 = (unsigned)(e - h + CHUNK - 1) / CHUNK;
      v = n0 | (n1 << 32);
    }
    packed[i] = v;
  }
}

// One warp per long row: its chunks in both phases; the row's slots (chunk partial
// sums, added in slot order when the row is finalised) are its phase-0 chunks, then
// its phase-1 chunks.
__global__ void k_long_chunks(int n_long, const int32_t* __restrict__ lrows, const int32_t* __restrict__ roffp,
                              const int32_t* __restrict__ hot_end, const unsigned long long* __restrict__ pre,
                              int4* __restrict__ ch0, int32_t* __restrict__ cl0, int4* __restrict__ ch1,
                              int32_t* __restrict__ cl1, int2* __restrict__ longs) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_long; i += (gridDim.x * blockDim.x) >> 5) {
    const int r = lrows[i];
    const int s0 = roffp[r], s1 = hot_end[r], s2 = roffp[r + 1];
    const unsigned long long p = pre[i], q = pre[i + 1];
    const int c0 = (int)(p & 0xffffffffull), c1 = (int)(p >> 32);
    const int n0 = (int)(q & 0xffffffffull) - c0, n1 = (int)(q >> 32) - c1;
    const int first = c0 + c1;
    if (lane == 0) longs[i] = make_int2(first, n0 + n1);
    for (int j = lane; j < n0; j += 32) {
      const int e = s0 + j * CHUNK;
      ch0[c0 + j] = make_int4(r, e, min(e + CHUNK, s1), first + j);
      cl0[c0 + j] = i;
    }
    for (int j = lane; j < n1; j += 32) {
      const int e = s1 + j * CHUNK;
      ch1[c1 + j] = make_int4(r, e, min(e + CHUNK, s2), first + n0 + j);
      cl1[c1 + j] = i;
    }
  }
}

__global__ void k_hot_end(int V, const int32_t* __restrict__ roffp, const int32_t* __restrict__ radjp, int hot,
                          int32_t* __restrict__ hot_end) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < V; r += gridDim.x * blockDim.x) {
    int lo = roffp[r], hi = roffp[r + 1];
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (radjp[m] < hot) lo = m + 1; else hi = m;
    }
    hot_end[r] = lo;
  }
}

__global__ void k_unpermute(int V, const int32_t* __restrict__ new_id, const float* __restrict__ src,
                            float* __restrict__ dst) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) dst[v] = src[new_id[v]];
}

__global__ void k_init(int V, const int32_t* __restrict__ odeg, float* __restrict__ pr, float* __restrict__ con,
                       State* st) {
  const float numNodes = (float)V;
  const float p0 = 1.0f / numNodes;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    pr[v] = p0;
    const int od = odeg[v];
    con[v] = od > 0 ? __fdiv_rn(p0, (float)od) : 0.0f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->done = 0;
    st->ticket = 0;
    st->diff = 0;
    st->extra = 0;
  }
}

// Warm start (sp_pagerank_dynamic): the caller's ranks, staged in `init` in the
// caller's vertex order, placed at their relabelled ids with their contributions.
__global__ void k_init_from(int V, const int32_t* __restrict__ new_id, const int32_t* __restrict__ odeg,
                            const float* __restrict__ init, float* __restrict__ pr, float* __restrict__ con,
                            State* st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int k = new_id[v];
    const float x = init[v];
    pr[k] = x;
    const int od = odeg[k];
    con[k] = od > 0 ? __fdiv_rn(x, (float)od) : 0.0f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->done = 0;
    st->ticket = 0;
    st->diff = 0;
    st->extra = 0;
  }
}

// Split run (sp_pagerank_part_begin): pr = 1/V and contrib at every id of the plan (the
// pads of the last positions have out-degree 0), so every part starts from the same
// full contrib vector without an exchange.
__global__ void k_init_part(int Vp, int V, const int32_t* __restrict__ odeg, float* __restrict__ pr,
                            float* __restrict__ con, State* st) {
  const float p0 = 1.0f / (float)V;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < Vp; v += gridDim.x * blockDim.x) {
    pr[v] = p0;
    const int od = odeg[v];
    con[v] = od > 0 ? __fdiv_rn(p0, (float)od) : 0.0f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->done = 0;
    st->ticket = 0;
    st->diff = 0;
    st->extra = 0;
  }
}

// Split run: once the caller has summed every part's diff into *diff, the stop test of
// the single-GPU run (iterate while diff > beta and fewer than max_iter iterations).
__global__ void k_decide(State* st, const double* __restrict__ diff, double beta, int max_iter) {
  if (st->done) return;
  const double d = *diff;
  st->diff = d;
  st->done = (d > beta && st->iter < max_iter) ? 0 : 1;
}

// ---- plain variant: the generated CUDA form (one thread per vertex, serial gather
// of pr[u]/outdeg(u), atomic float diff; backend_cuda/dsl_cpp_generator.cpp:1682-1761)
__global__ void k_plain_iter(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ roff,
                             const int32_t* __restrict__ radj, const float* __restrict__ pr,
                             float* __restrict__ prn, float base, float delta, float* diff) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  float sum = 0.0f;
  for (int e = roff[v]; e < roff[v + 1]; ++e) {
    const int u = radj[e];
    sum = sum + pr[u] / (float)(off[u + 1] - off[u]);
  }
  const float np = base + delta * sum;
  atomicAdd(diff, fabsf(np - pr[v]));
  prn[v] = np;
}

__global__ void k_plain_init(int V, float* pr) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) pr[v] = 1.0f / (float)V;
}

}  // namespace pr

// Relabel vertices by out-degree (descending, stable) and build the reverse CSR in the
// new ids with every row ascending, all on the device. The rows come from a stable
// transpose: the (new dst, new src) pair of every edge, written in ascending source
// order from the forward CSR and radix-sorted by dst (LSD radix sort keeps equal keys
// in input order, so each row's sources stay ascending). Also lays out the per-graph
// iteration buffers.
static int relabel(sp_graph* g, PrPlan* p) {
  const int V = g->V;
  const int E = (int)g->E;
  const int np = p->nparts, S = p->S, Vp = p->Vp;  // ids: lay(rank) in [0, Vp)
  cudaStream_t s = g->stream;
  Arena& A = p->graph_mem;
  A.want(p->new_id, V);
  A.want(p->od, Vp);
  A.want(p->roffp, (size_t)Vp + 1);
  A.want(p->radjp, (size_t)E);
  A.want(p->outbuf, V);
  A.want(p->hot_end, Vp);
  A.want(p->part, Vp);
  A.want(p->diff_part, 2 * (size_t)num_sms() * 32);
  A.want(p->state, 1);
  for (int i = 0; i < 2; ++i) {
    A.want(p->prb[i], Vp);
    A.want(p->con[i], Vp);
  }
  SP_TRY(A.commit());

  int bits = 1;
  while (bits < 31 && (1 << bits) < Vp) ++bits;
  size_t t_vsort = 0, t_scan = 0, t_esort = 0;
  cub::DoubleBuffer<int32_t> nk(nullptr, nullptr), nv(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, t_vsort, (const int32_t*)nullptr, (int32_t*)nullptr,
                                  (const int32_t*)nullptr, (int32_t*)nullptr, V, 0, 32, s);
  cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (const int32_t*)nullptr, (int32_t*)nullptr, V + 1, s);
  cub::DeviceRadixSort::SortPairs(nullptr, t_esort, nk, nv, E, 0, bits, s);
  Arena T;
  dspan<int32_t> key, id, skey, inv, offp, dst, dst_alt, src, big, odk;
  dspan<int> nbig;
  dspan<unsigned char> temp;
  T.want(odk, V);  // out-degrees in rank order (the transpose's source order)
  T.want(key, V);
  T.want(id, V);
  T.want(skey, V);
  T.want(inv, V);
  T.want(offp, V);
  T.want(dst, E);
  T.want(dst_alt, E);
  T.want(src, E);
  T.want(big, V);
  T.want(nbig, 1);
  T.want(temp, std::max(t_vsort, std::max(t_scan, t_esort)));
  SP_TRY(T.commit());
  const size_t tb = temp.n;

  const int grid = num_sms() * 8;
  pr::k_deg_keys<<<grid, 256, 0, s>>>(V, p->order, g->off.p, g->roff.p, key.p, id.p);
  SP_CHECK_LAUNCH();
  size_t t = tb;
  SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, key.p, skey.p, id.p, inv.p, V, 0, 32, s));
  pr::k_relabel_rows<<<grid, 256, 0, s>>>(V, np, S, inv.p, g->off.p, p->new_id.p, odk.p);
  SP_CHECK_LAUNCH();
  t = tb;
  SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, t, odk.p, offp.p, V, s));
  SP_CHECK_CUDA(cudaMemsetAsync(nbig.p, 0, sizeof(int), s));
  pr::k_fwd_pairs<<<grid, 256, 0, s>>>(V, np, S, inv.p, p->new_id.p, g->off.p, g->adj.p, offp.p, odk.p, dst.p,
                                       src.p, big.p, nbig.p);
  SP_CHECK_LAUNCH();
  pr::k_fwd_pairs_big<<<num_sms() * 8, 256, 0, s>>>(np, S, inv.p, p->new_id.p, g->off.p, g->adj.p, offp.p, odk.p,
                                                     dst.p, src.p, big.p, nbig.p);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemsetAsync(p->od.p, 0, sizeof(int32_t) * Vp, s));
  pr::k_od_layout<<<grid, 256, 0, s>>>(V, np, S, odk.p, p->od.p);
  SP_CHECK_LAUNCH();
  cub::DoubleBuffer<int32_t> keys(dst.p, dst_alt.p), vals(src.p, p->radjp.p);
  t = tb;
  SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, keys, vals, E, 0, bits, s));
  if (E > 0 && vals.Current() != p->radjp.p)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->radjp.p, vals.Current(), sizeof(int32_t) * E, cudaMemcpyDeviceToDevice, s));
  // row offsets of the relabelled reverse CSR straight from the sorted destinations
  // (no reverse CSR of the caller's graph is needed)
  SP_TRY(offsets_of_sorted(Vp, E, keys.Current(), p->roffp.p, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  return SP_OK;
}

// Row classes and long-row chunks for one hot setting, built on the device: a stable
// 3-bit radix sort groups each phase's rows by class (ascending ids within a class),
// and one scan over the long rows places their chunks and chunk-partial slots. The
// host reads back only the class sizes and the chunk totals.
static int build_pr_plan(sp_graph* g, int hot, int order, int part = 0, int nparts = 1) {
  if (g->pr && g->pr->hot == hot && g->pr->order == order && g->pr->part_idx == part && g->pr->nparts == nparts)
    return SP_OK;
  if (order != 0) SP_TRY(ensure_reverse(g));  // in-degree classes read the caller's reverse offsets
  if (g->pr && (g->pr->order != order || g->pr->part_idx != part || g->pr->nparts != nparts)) {
    free_pr_plan(g->pr);  // a new vertex order or split: a new plan
    g->pr = nullptr;
  }
  PrPlan* p = g->pr;
  if (!p) {
    p = new PrPlan();
    p->order = order;
    p->nparts = nparts;
    p->part_idx = part;
    p->S = nparts == 1 ? g->V : (g->V + nparts - 1) / nparts;
    p->Vp = nparts == 1 ? g->V : nparts * p->S;
    p->lo = nparts == 1 ? 0 : part * p->S;
    p->hi = nparts == 1 ? g->V : p->lo + (g->V - part + nparts - 1) / nparts;  // ranks k = part mod nparts
    int st = relabel(g, p);
    if (st) {
      free_pr_plan(p);
      return st;
    }
    g->pr = p;
  }
  cudaStream_t s = g->stream;
  p->pend_iters = 0;
  if (p->exec) {  // it refers to the buffers rebuilt below
    cudaGraphExecDestroy(p->exec);
    p->exec = nullptr;
  }
  p->hot = -1;  // incomplete until the end
  const int V = p->Vp;  // rows of the plan's id space
  const int32_t* hend = p->roffp.p;  // hot = 0: every row is all cold
  if (hot > 0) {
    pr::k_hot_end<<<num_sms() * 8, 256, 0, s>>>(V, p->roffp.p, p->radjp.p, hot, p->hot_end.p);
    SP_CHECK_LAUNCH();
    hend = p->hot_end.p;
  }

  size_t t_sort = 0, t_scan = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (const uint8_t*)nullptr, (uint8_t*)nullptr,
                                  (const int32_t*)nullptr, (int32_t*)nullptr, V, 0, 3, s);
  cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                V + 1, s);
  Arena T;
  dspan<uint8_t> key0, key1, skey;
  dspan<int32_t> iota;
  dspan<int> counts;
  dspan<unsigned long long> packed, pre;
  dspan<unsigned char> temp;
  T.want(key0, V);
  T.want(key1, V);
  T.want(skey, V);
  T.want(iota, V);
  T.want(counts, 2 * pr::N_CLASS);
  T.want(packed, (size_t)V + 1);
  T.want(pre, (size_t)V + 1);
  T.want(temp, std::max(t_sort, t_scan));
  SP_TRY(T.commit());
  const size_t tb = temp.n;

  SP_CHECK_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * 2 * pr::N_CLASS, s));
  pr::k_row_classes<<<num_sms() * 8, 256, 0, s>>>(V, p->lo, p->hi, p->roffp.p, hend, key0.p, key1.p, iota.p,
                                                   counts.p);
  SP_CHECK_LAUNCH();
  int hc[2 * pr::N_CLASS];
  SP_TRY(copy_out(hc, counts.p, sizeof(hc), s));
  int n_rows[2] = {0, 0};
  for (int ph = 0; ph < 2; ++ph) {
    const int* c = hc + ph * pr::N_CLASS;
    p->row_base[ph][0] = p->task_base[ph][0] = 0;
    for (int k = 0; k < 4; ++k) {
      const int per = 32 / pr::BIN_W[k];
      p->row_base[ph][k + 1] = p->row_base[ph][k] + c[k];
      p->task_base[ph][k + 1] = p->task_base[ph][k] + (c[k] + per - 1) / per;
    }
    n_rows[ph] = p->row_base[ph][4];
  }
  p->n_long = hc[pr::N_CLASS + 5];
  p->n_zero = hc[pr::N_CLASS + 6];
  const int long_at = V - p->n_long - p->n_zero;  // classes 5 and 6 sort last
  // a segment of h edges has at most h / CHUNK + 1 chunks
  const size_t max_chunks = (size_t)(g->E / pr::CHUNK) + (size_t)p->n_long + 1;

  Arena& B = p->bin_mem;
  B.want(p->rows[0], n_rows[0] ? V : 1);
  B.want(p->rows[1], V);
  for (int ph = 0; ph < 2; ++ph) {
    B.want(p->chunks[ph], p->n_long ? max_chunks : 1);
    B.want(p->chunk_long[ph], p->n_long ? max_chunks : 1);
  }
  B.want(p->longs, std::max(1, p->n_long));
  B.want(p->long_ctr, std::max(1, p->n_long));
  B.want(p->chunk_part, p->n_long ? 2 * max_chunks : 1);
  SP_TRY(B.commit());

  size_t t = tb;
  SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, key1.p, skey.p, iota.p, p->rows[1].p, V, 0, 3, s));
  if (n_rows[0]) {
    t = tb;
    SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, key0.p, skey.p, iota.p, p->rows[0].p, V, 0, 3, s));
  }
  p->n_chunks[0] = p->n_chunks[1] = 0;
  if (p->n_long) {
    const int32_t* lrows = p->rows[1].p + long_at;
    pr::k_long_counts<<<num_sms() * 2, 256, 0, s>>>(p->n_long, lrows, p->roffp.p, hend, packed.p);
    SP_CHECK_LAUNCH();
    t = tb;
    SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, t, packed.p, pre.p, p->n_long + 1, s));
    unsigned long long tot = 0;
    SP_TRY(copy_out(&tot, pre.p + p->n_long, sizeof(tot), s));
    p->n_chunks[0] = (int)(tot & 0xffffffffull);
    p->n_chunks[1] = (int)(tot >> 32);
    if ((size_t)p->n_chunks[0] > max_chunks || (size_t)p->n_chunks[1] > max_chunks) {
      set_error("pagerank plan: %d/%d chunks above the bound %zu", p->n_chunks[0], p->n_chunks[1], max_chunks);
      return SP_ERR_UNSUPPORTED;
    }
    pr::k_long_chunks<<<num_sms() * 2, 256, 0, s>>>(p->n_long, lrows, p->roffp.p, hend, pre.p, p->chunks[0].p,
                                                     p->chunk_long[0].p, p->chunks[1].p, p->chunk_long[1].p,
                                                     p->longs.p);
    SP_CHECK_LAUNCH();
  }
  SP_CHECK_CUDA(cudaMemsetAsync(p->long_ctr.p, 0, sizeof(unsigned int) * std::max(1, p->n_long), s));
  p->zrows = p->rows[1].p + long_at + p->n_long;
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  p->hot = hot;
  return SP_OK;
}

// The iteration kernel's arguments for plan p (V = the graph's vertices, for the base
// term (1 - delta) / V).
static pr::IterArgs iter_args(const PrPlan* p, float beta, float delta, int n_iter, int V) {
  pr::IterArgs a;
  a.roff = p->roffp.p;
  a.radj = p->radjp.p;
  a.hot_end = p->hot > 0 ? p->hot_end.p : p->roffp.p;  // hot = 0: each row's split is its start
  a.od = p->od.p;
  a.longs = p->longs.p;
  a.long_ctr = p->long_ctr.p;
  a.chunk_part = p->chunk_part.p;
  a.part = p->part.p;
  a.diff_part = p->diff_part.p;
  a.st = p->state.p;
  for (int ph = 0; ph < 2; ++ph) {
    a.ph[ph].rows = p->rows[ph].p;
    a.ph[ph].chunks = p->chunks[ph].p;
    a.ph[ph].chunk_long = p->chunk_long[ph].p;
    for (int k = 0; k < 5; ++k) {
      a.ph[ph].row_base[k] = p->row_base[ph][k];
      a.ph[ph].task_base[k] = p->task_base[ph][k];
    }
    a.ph[ph].n_chunks = p->n_chunks[ph];
  }
  a.delta = delta;
  a.base = (1.0f - delta) / (float)V;
  a.beta = (double)beta;
  a.max_iter = n_iter;
  a.two_phase = p->two_phase() ? 1 : 0;
  a.l1_hot = 0;
  a.diff_out = nullptr;
  return a;
}

// ---- learned kernel variant -------------------------------------------------------
// The table the variant model scores: how many of the most-gathered sources allocate
// their contrib gathers in L1 (0 = all), the srcList L1 policy, and 16-byte srcList loads.
// Entry 10 is the fixed default (32768, evict-first, 4-byte loads).
namespace pr {
struct Variant {
  int l1_hot, src_hint, vec;
};
constexpr Variant VARIANTS[] = {{0, 0, 0},      {0, 2, 0},      {0, 2, 1},      {8192, 0, 0},
                                {8192, 2, 0},   {8192, 2, 1},   {16384, 2, 0},  {32768, 0, 0},
                                {32768, 0, 1},  {32768, 2, 1},  {32768, 2, 0},  {65536, 2, 0},
                                {131072, 0, 0}, {131072, 2, 0}, {131072, 2, 1}, {524288, 2, 0}};
constexpr int N_VARIANTS = (int)(sizeof(VARIANTS) / sizeof(VARIANTS[0]));
constexpr int DEFAULT_VARIANT = 10;
constexpr int SHARE_K[3] = {8192, 32768, 131072};

// sums of od[0 .. SHARE_K[j]) (od is the out-degree in relabelled order, descending);
// the kernel spells out SHARE_K's three values
__global__ void k_top_share(int V, const int32_t* __restrict__ od, unsigned long long* out) {
  __shared__ unsigned long long s[3];
  if (threadIdx.x < 3) s[threadIdx.x] = 0;
  __syncthreads();
  unsigned long long a[3] = {0, 0, 0};
  const int lim = min(V, 131072);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
    const unsigned long long d = (unsigned long long)od[i];
    if (i < 8192) a[0] += d;
    if (i < 32768) a[1] += d;
    a[2] += d;
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const unsigned long long w = warp_sum(a[j]);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&s[j], w);
  }
  __syncthreads();
  if (threadIdx.x < 3 && s[threadIdx.x]) atomicAdd(&out[threadIdx.x], s[threadIdx.x]);
}
}  // namespace pr

int pr_variant_count() { return pr::N_VARIANTS; }

static int pr_plan_for_call(sp_graph* g) {
  const int hot = std::max(0, std::min(g->pr_hot >= 0 ? g->pr_hot : pr::HOT_DEFAULT, pr::HOT_MAX));
  const int order = g->pr_order >= 0 ? g->pr_order : pr::ORDER_DEFAULT;
  return build_pr_plan(g, hot, order);
}

static int pr_variant_stats(sp_graph* g) {
  PrPlan* p = g->pr;
  if (p->vorder == p->order) return SP_OK;
  cudaStream_t s = g->stream;
  dbuf<unsigned long long> acc;
  SP_TRY(acc.alloc(3));
  SP_CHECK_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(unsigned long long) * 3, s));
  pr::k_top_share<<<std::max(1, std::min(num_sms(), (g->V + 255) / 256)), 256, 0, s>>>(g->V, p->od.p, acc.p);
  SP_CHECK_LAUNCH();
  unsigned long long h[3];
  SP_TRY(copy_out(h, acc.p, sizeof(h), s));
  DegStats ds;
  SP_TRY(degree_stats(p->roffp.p, g->V, nullptr, 0, s, &ds));
  const double E = std::max<double>(1.0, (double)g->E);
  for (int j = 0; j < 3; ++j) p->vshare[j] = (double)h[j] / E;
  p->vin_max = ds.max_deg;
  p->vin_sq = ds.sum_sq;
  p->vorder = p->order;
  return SP_OK;
}

// Inputs: graph shape over in-degrees (the pull's rows), the hot shares, then the
// candidate: log of the sources that allocate in L1, that count as a fraction of V,
// srcList policy, vector loads, and the share of gathers that hit those sources.
int pr_variant_features(sp_graph* g, int cand, float* x, int* applicable) {
  if (cand < 0 || cand >= pr::N_VARIANTS) return SP_ERR_INVALID;
  SP_TRY(pr_plan_for_call(g));
  SP_TRY(pr_variant_stats(g));
  const PrPlan* p = g->pr;
  const pr::Variant& c = pr::VARIANTS[cand];
  const double V = g->V, E = (double)g->E, avg = E / std::max(1.0, V), mx = (double)p->vin_max;
  const double eff = c.l1_hot == 0 ? V : std::min<double>(c.l1_hot, V);
  double share = 1.0;  // share of gathers from the first eff sources
  if (eff < V) {
    share = eff <= pr::SHARE_K[0] ? p->vshare[0] * eff / pr::SHARE_K[0]
            : eff <= pr::SHARE_K[1]
                ? p->vshare[0] + (p->vshare[1] - p->vshare[0]) * (eff - pr::SHARE_K[0]) / (pr::SHARE_K[1] - pr::SHARE_K[0])
            : eff <= pr::SHARE_K[2]
                ? p->vshare[1] + (p->vshare[2] - p->vshare[1]) * (eff - pr::SHARE_K[1]) / (pr::SHARE_K[2] - pr::SHARE_K[1])
                : p->vshare[2] + (1.0 - p->vshare[2]) * (eff - pr::SHARE_K[2]) / std::max(1.0, V - pr::SHARE_K[2]);
    share = std::min(1.0, share);
  }
  x[0] = (float)std::log2(std::max(1.0, V));
  x[1] = (float)std::log2(E + 1.0);
  x[2] = (float)avg;
  x[3] = (float)std::log2(mx + 1.0);
  x[4] = (float)std::log2(((double)p->vin_sq / std::max(1.0, E)) + 1.0);  // in-degree second moment
  x[5] = (float)p->vshare[0];
  x[6] = (float)p->vshare[1];
  x[7] = (float)p->vshare[2];
  x[8] = (float)std::log2(eff + 1.0);
  x[9] = (float)(eff / std::max(1.0, V));
  x[10] = (float)c.src_hint * 0.5f;
  x[11] = (float)c.vec;
  x[12] = (float)share;
  *applicable = 1;
  return SP_OK;
}

// The candidate this call runs: forced by "pr.variant", else learned when a model is
// loaded and no variant knob is set; -1 = the knobs and defaults.
static int pr_variant_pick(sp_graph* g, int* cand) {
  *cand = -1;
  const int mode = g->variant[VAR_PR];
  if (mode >= 0) {
    *cand = mode;
    return SP_OK;
  }
  if (mode != -1 || g->pr_l1_hot >= 0 || g->pr_src_hint >= 0 || g->pr_vec >= 0) return SP_OK;
  const unsigned gen = variant_generation(VAR_PR);
  if (!gen) return SP_OK;
  PrPlan* p = g->pr;
  if (p->var_gen == gen && p->var_choice >= 0) {
    *cand = p->var_choice;
    return SP_OK;
  }
  std::vector<float> X((size_t)pr::N_VARIANTS * SP_MLP_IN);
  std::vector<int> ok(pr::N_VARIANTS);
  for (int k = 0; k < pr::N_VARIANTS; ++k) SP_TRY(pr_variant_features(g, k, X.data() + (size_t)k * SP_MLP_IN, &ok[k]));
  int best = -1;
  const int st = variant_choose(VAR_PR, X, ok, pr::DEFAULT_VARIANT, g->stream, &best);
  if (st == SP_ERR_UNSUPPORTED) return SP_OK;  // unloaded meanwhile
  SP_TRY(st);
  p->var_choice = best;
  p->var_gen = gen;
  *cand = best;
  return SP_OK;
}

// init: starting ranks in the caller's vertex order (host or device), or null for 1/V.
static int pr_tuned(sp_graph* g, float beta, float delta, int32_t maxIter, float* out, int32_t* iters,
                    double* fdiff, const float* init = nullptr) {
  const int hot = std::max(0, std::min(g->pr_hot >= 0 ? g->pr_hot : pr::HOT_DEFAULT, pr::HOT_MAX));
  const int order = g->pr_order >= 0 ? g->pr_order : pr::ORDER_DEFAULT;
  SP_TRY(build_pr_plan(g, hot, order));
  PrPlan* p = g->pr;
  cudaStream_t s = g->stream;
  const int V = g->V;
  const int n_iter = std::max(1, (int)maxIter);
  pr::IterArgs a = iter_args(p, beta, delta, n_iter, V);
  int per_sm = 0;
  int sh = g->pr_src_hint >= 0 ? g->pr_src_hint : pr::SRC_HINT_DEFAULT;
  int l1_hot = g->pr_l1_hot >= 0 ? g->pr_l1_hot : pr::L1_HOT_DEFAULT;
  int vec = g->pr_vec >= 0 ? g->pr_vec : pr::VEC_DEFAULT;
  int cand = -1;
  SP_TRY(pr_variant_pick(g, &cand));
  if (cand >= 0) {
    sh = pr::VARIANTS[cand].src_hint;
    l1_hot = pr::VARIANTS[cand].l1_hot;
    vec = pr::VARIANTS[cand].vec;
  }
  g->last_variant[VAR_PR] = cand;
  a.l1_hot = l1_hot;
  const int gh = l1_hot > 0 ? 1 : 0;
  using PhaseFn = void (*)(pr::IterArgs, const float*, const float*, float*, float*);
  static const PhaseFn table[3][2][2] = {
      {{pr::k_phase<1, 0, 0, 0>, pr::k_phase<1, 0, 0, 1>}, {pr::k_phase<1, 0, 1, 0>, pr::k_phase<1, 0, 1, 1>}},
      {{pr::k_phase<1, 1, 0, 0>, pr::k_phase<1, 1, 0, 1>}, {pr::k_phase<1, 1, 1, 0>, pr::k_phase<1, 1, 1, 1>}},
      {{pr::k_phase<1, 2, 0, 0>, pr::k_phase<1, 2, 0, 1>}, {pr::k_phase<1, 2, 1, 0>, pr::k_phase<1, 2, 1, 1>}}};
  const PhaseFn ph1 = table[sh][gh][vec];
  const int exec_key = sh | (vec << 2) | (l1_hot << 3);
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ph1, pr::THREADS, 0));
  const int grid = std::max(1, std::min(num_sms() * 32, num_sms() * std::max(1, per_sm)));
  if (init) {
    SP_CHECK_CUDA(cudaMemcpyAsync(p->outbuf.p, init, sizeof(float) * V, cudaMemcpyDefault, s));
    pr::k_init_from<<<num_sms() * 4, 256, 0, s>>>(V, p->new_id.p, p->od.p, p->outbuf.p, p->prb[0].p, p->con[0].p,
                                                  p->state.p);
  } else {
    pr::k_init<<<num_sms() * 4, 256, 0, s>>>(V, p->od.p, p->prb[0].p, p->con[0].p, p->state.p);
  }
  SP_CHECK_LAUNCH();
  // the iterations: every kernel returns at once after the stop test has ended the run
  auto enqueue = [&](cudaStream_t cs) {
    for (int k = 0; k < n_iter; ++k) {
      const int c = k & 1, n = c ^ 1;
      if (k < 2 && p->n_zero)
        pr::k_zero_rows<<<num_sms() * 2, 256, 0, cs>>>(a, p->zrows, p->n_zero, p->prb[c].p, p->prb[n].p, p->con[n].p);
      if (a.two_phase)
        pr::k_phase<0, 1, 0, 0><<<grid, pr::THREADS, 0, cs>>>(a, p->prb[c].p, p->con[c].p, p->prb[n].p, p->con[n].p);
      ph1<<<grid, pr::THREADS, 0, cs>>>(a, p->prb[c].p, p->con[c].p, p->prb[n].p, p->con[n].p);
    }
  };
  const bool cached = p->exec && p->exec_iters == n_iter && p->exec_beta == beta && p->exec_delta == delta &&
                      p->exec_sh == exec_key;
  const bool repeat = p->pend_iters == n_iter && p->pend_beta == beta && p->pend_delta == delta &&
                      p->pend_sh == exec_key;
  if (!cached && !repeat) {
    // first call with these settings: launch directly (no capture and instantiation
    // before the first kernel runs); a call that repeats them captures the graph
    enqueue(s);
    SP_CHECK_LAUNCH();
    p->pend_iters = n_iter;
    p->pend_beta = beta;
    p->pend_delta = delta;
    p->pend_sh = exec_key;
  } else if (!cached) {
    if (p->exec) {
      cudaGraphExecDestroy(p->exec);
      p->exec = nullptr;
    }
    if (!p->cap) SP_CHECK_CUDA(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
    cudaStream_t cs = p->cap;  // capture only records: nothing runs on it
    cudaGraph_t graph;
    SP_CHECK_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    enqueue(cs);
    cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    if (ce != cudaSuccess) {
      set_error("pagerank graph capture: %s", cudaGetErrorString(ce));
      return SP_ERR_CUDA;
    }
    ce = cudaGraphInstantiate(&p->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      p->exec = nullptr;
      set_error("pagerank graph instantiate: %s", cudaGetErrorString(ce));
      return SP_ERR_CUDA;
    }
    p->exec_iters = n_iter;
    p->exec_beta = beta;
    p->exec_delta = delta;
    p->exec_sh = exec_key;
  }
  if (cached || repeat) SP_CHECK_CUDA(cudaGraphLaunch(p->exec, s));
  g_launches.fetch_add((unsigned long long)n_iter * (p->two_phase() ? 2 : 1) +
                       (p->n_zero ? std::min(2, n_iter) : 0));
  pr::State st;
  SP_TRY(copy_out(&st, p->state.p, sizeof(st), s));
  if (out) {
    pr::k_unpermute<<<num_sms() * 4, 256, 0, s>>>(V, p->new_id.p, p->prb[st.iter & 1].p, p->outbuf.p);
    SP_CHECK_LAUNCH();
    SP_TRY(copy_out(out, p->outbuf.p, sizeof(float) * V, s));
  }
  if (iters) *iters = st.iter;
  if (fdiff) *fdiff = st.diff;
  return SP_OK;
}

static int pr_plain(sp_graph* g, float beta, float delta, int32_t maxIter, float* out, int32_t* iters,
                    double* fdiff) {
  SP_TRY(ensure_reverse(g));
  cudaStream_t s = g->stream;
  const int V = g->V;
  dbuf<float> d_diff, b0, b1;
  SP_TRY(d_diff.alloc(1));
  SP_TRY(b0.alloc(V));
  SP_TRY(b1.alloc(V));
  float* prb[2] = {b0.p, b1.p};
  const int tb = 512;  // the generator's launch shape (backend_cuda/dsl_cpp_generator.cpp:56-77)
  const int nb = (V + tb - 1) / tb;
  pr::k_plain_init<<<nb, tb, 0, s>>>(V, prb[0]);
  SP_CHECK_LAUNCH();
  const float base = (1.0f - delta) / (float)V;
  int it = 0;
  float diff = 0;
  int cur = 0;
  do {
    SP_CHECK_CUDA(cudaMemsetAsync(d_diff.p, 0, sizeof(float), s));
    pr::k_plain_iter<<<nb, tb, 0, s>>>(V, g->off.p, g->roff.p, g->radj.p, prb[cur], prb[cur ^ 1], base, delta,
                                        d_diff.p);
    SP_CHECK_LAUNCH();
    SP_TRY(copy_out(&diff, d_diff.p, sizeof(float), s));
    cur ^= 1;
    ++it;
  } while (diff > beta && it < maxIter);
  if (out) SP_TRY(copy_out(out, prb[cur], sizeof(float) * V, s));
  if (iters) *iters = it;
  if (fdiff) *fdiff = diff;
  return SP_OK;
}

}  // namespace sp

extern "C" int sp_pagerank(sp_graph_h g, float beta, float delta, int32_t maxIter, float* pageRank,
                           int32_t* iterations, double* final_diff, int32_t variant) {
  if (!g) {
    sp::set_error("sp_pagerank: NULL graph");
    return SP_ERR_INVALID;
  }
  if (variant == SP_PR_PLAIN) return sp::pr_plain(g, beta, delta, maxIter, pageRank, iterations, final_diff);
  if (variant != SP_PR_TUNED) {
    sp::set_error("sp_pagerank: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  return sp::pr_tuned(g, beta, delta, maxIter, pageRank, iterations, final_diff);
}

// DynPR's Batch block (dynamicDSLCodes/dynamicBatchPR:112-153): the batch is applied
// (deletions, then additions), then PageRank runs from the caller's ranks instead of
// 1/V, with the static form's iteration and stop test.
extern "C" int sp_pagerank_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src,
                                   const int32_t* dst, const int32_t* weight, float beta, float delta,
                                   int32_t maxIter, float* pageRank, int32_t* iterations, double* final_diff) {
  using namespace sp;
  if (!g || !pageRank || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_pagerank_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  if (n > 0) SP_TRY(update_graph(g, n, type, src, dst, weight));
  return pr_tuned(g, beta, delta, maxIter, pageRank, iterations, final_diff, pageRank);
}

// ---- PageRank split over GPUs by vertices (one part per rank) ----------------------
// Replaces the host-staged exchange of the reference's multi-GPU generator
// (backend_multigpu/dsl_cpp_generator.cpp:604-678): part r owns the rows of ids
// [r * S, r * S + count_r) of a split plan (lay()), computes their ranks and contrib
// each iteration, and the caller all-gathers the contrib slices (S floats per part)
// and sums the parts' diffs with its collectives, on the device, between the calls.
namespace sp {
static int part_plan(sp_graph* g, const char* who, PrPlan** out) {
  if (!g || !g->pr || g->pr->nparts < 1 || !g->pr->pcon[0]) {
    set_error("%s: no split PageRank begun on this graph", who);
    return SP_ERR_INVALID;
  }
  *out = g->pr;
  return SP_OK;
}
}  // namespace sp

extern "C" int sp_pagerank_part_begin(sp_graph_h g, int32_t part, int32_t nparts, float beta, float delta,
                                      int32_t maxIter, float* con0, float* con1, double* diff, int32_t* slice) {
  using namespace sp;
  if (!g || nparts < 1 || part < 0 || part >= nparts || !con0 || !con1 || !diff || !slice) {
    set_error("sp_pagerank_part_begin: invalid argument");
    return SP_ERR_INVALID;
  }
  if (g->V == 0) {
    set_error("sp_pagerank_part_begin: empty graph");
    return SP_ERR_INVALID;
  }
  SP_TRY(build_pr_plan(g, 0, 0, part, nparts));
  PrPlan* p = g->pr;
  p->pcon[0] = con0;
  p->pcon[1] = con1;
  p->pdiff = diff;
  p->pbeta = beta;
  p->pdelta = delta;
  p->pmax_iter = std::max(1, (int)maxIter);  // the DSL's do-while runs at least once
  pr::k_init_part<<<num_sms() * 4, 256, 0, g->stream>>>(p->Vp, g->V, p->od.p, p->prb[0].p, con0, p->state.p);
  SP_CHECK_LAUNCH();
  *slice = p->S;
  return SP_OK;
}

extern "C" int sp_pagerank_part_iterate(sp_graph_h g, int32_t k) {
  using namespace sp;
  PrPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_pagerank_part_iterate", &p));
  if (k < 0) {
    set_error("sp_pagerank_part_iterate: iteration %d", k);
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  // no local stop: the part's kernel only counts the iteration; k_decide applies the
  // stop test to the summed diff
  pr::IterArgs a = iter_args(p, -1.0f, p->pdelta, INT_MAX, g->V);
  a.diff_out = p->pdiff;
  const int sh = g->pr_src_hint >= 0 ? g->pr_src_hint : pr::SRC_HINT_DEFAULT;
  using PhaseFn = void (*)(pr::IterArgs, const float*, const float*, float*, float*);
  const PhaseFn ph1 = sh == 1 ? pr::k_phase<1, 1, 0, 0> : sh == 2 ? pr::k_phase<1, 2, 0, 0> : pr::k_phase<1, 0, 0, 0>;
  int per_sm = 0;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ph1, pr::THREADS, 0));
  const int grid = std::max(1, std::min(num_sms() * 32, num_sms() * std::max(1, per_sm)));
  const int c = k & 1, n = c ^ 1;
  if (k < 2 && p->n_zero) {
    pr::k_zero_rows<<<num_sms() * 2, 256, 0, s>>>(a, p->zrows, p->n_zero, p->prb[c].p, p->prb[n].p, p->pcon[n]);
    SP_CHECK_LAUNCH();
  }
  ph1<<<grid, pr::THREADS, 0, s>>>(a, p->prb[c].p, p->pcon[c], p->prb[n].p, p->pcon[n]);
  SP_CHECK_LAUNCH();
  return SP_OK;
}

extern "C" int sp_pagerank_part_decide(sp_graph_h g) {
  using namespace sp;
  PrPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_pagerank_part_decide", &p));
  pr::k_decide<<<1, 1, 0, g->stream>>>(p->state.p, p->pdiff, (double)p->pbeta, p->pmax_iter);
  SP_CHECK_LAUNCH();
  return SP_OK;
}

extern "C" int sp_pagerank_part_state(sp_graph_h g, int32_t* iterations, int32_t* done, double* diff) {
  using namespace sp;
  PrPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_pagerank_part_state", &p));
  pr::State st;
  SP_TRY(copy_out(&st, p->state.p, sizeof(st), g->stream));
  if (iterations) *iterations = st.iter;
  if (done) *done = st.done;
  if (diff) *diff = st.diff;
  return SP_OK;
}

extern "C" int sp_pagerank_part_ranks(sp_graph_h g, float* slice) {
  using namespace sp;
  PrPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_pagerank_part_ranks", &p));
  if (!slice) {
    set_error("sp_pagerank_part_ranks: NULL slice");
    return SP_ERR_INVALID;
  }
  pr::State st;
  SP_TRY(copy_out(&st, p->state.p, sizeof(st), g->stream));
  return copy_out(slice, p->prb[st.iter & 1].p + p->lo, sizeof(float) * p->S, g->stream);
}

extern "C" int sp_pagerank_part_finish(sp_graph_h g, const float* ranks, float* pageRank) {
  using namespace sp;
  PrPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_pagerank_part_finish", &p));
  if (!ranks || !pageRank) {
    set_error("sp_pagerank_part_finish: NULL argument");
    return SP_ERR_INVALID;
  }
  pr::k_unpermute<<<num_sms() * 4, 256, 0, g->stream>>>(g->V, p->new_id.p, ranks, p->outbuf.p);
  SP_CHECK_LAUNCH();
  return copy_out(pageRank, p->outbuf.p, sizeof(float) * g->V, g->stream);
}
