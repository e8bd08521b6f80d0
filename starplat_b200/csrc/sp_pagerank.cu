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

struct Phase {
  const int32_t* __restrict__ rows;   // binned row ids
  const int4* __restrict__ tasks;     // warp tasks {W, start, count, 0}
  const int4* __restrict__ chunks;    // {row, e_begin, e_end, slot}
  const int32_t* __restrict__ chunk_long;  // long-row index of each chunk
  int n_tasks;
  int n_chunks;
};
}  // namespace pr

struct PrPlan {
  dbuf<int32_t> new_id;   // vertex -> rank by out-degree (descending, stable)
  dbuf<int32_t> od;       // out-degree, in relabelled order
  dbuf<int32_t> roffp, radjp;  // reverse CSR in relabelled ids, rows sorted
  dbuf<int32_t> hot_end;  // per row: first edge whose source id >= hot
  dbuf<float> outbuf;     // result in original vertex order
  dbuf<int32_t> rows[2], chunk_long[2], zrows;
  dbuf<int4> tasks[2], chunks[2];
  int n_tasks[2] = {0, 0}, n_chunks[2] = {0, 0}, n_zero = 0, n_long = 0;
  dbuf<int2> longs;       // [n_long] {first slot, slot count}
  dbuf<unsigned int> long_ctr;
  dbuf<double> chunk_part, part;
  dbuf<double> diff_part;
  dbuf<float> prb[2], con[2];
  dbuf<pr::State> state;
  int hot = -1;           // hot id count the plan was built for
  cudaGraphExec_t exec = nullptr;
  int exec_iters = 0;
  float exec_beta = -1, exec_delta = -1;
  cudaStream_t exec_stream = nullptr;
};

void free_pr_plan(PrPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
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

// srcList is read once per iteration: in the hot phase keep it out of L1 so the
// hot block of contrib stays resident.
template <int PH>
__device__ __forceinline__ int ld_src(const int32_t* p) {
  if (PH == 0) {
    int v;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
  }
  return __ldg(p);
}

// Sum of con[radj[i]] for i in [b, e) by a group of W lanes (sl = lane within the
// group), U loads in flight per lane per round, reduced with a fixed xor tree.
template <int PH, int W, int U>
__device__ __forceinline__ double group_row_sum(int b, int e, int sl, const int32_t* __restrict__ radj,
                                                const float* __restrict__ con) {
  double acc = 0;
  for (int base = b; base < e; base += W * U) {
    int idx[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int i = base + sl + W * k;
      idx[k] = i < e ? ld_src<PH>(radj + i) : -1;
    }
    float v[U];
#pragma unroll
    for (int k = 0; k < U; ++k) v[k] = idx[k] >= 0 ? __ldg(con + idx[k]) : 0.0f;
#pragma unroll
    for (int k = 0; k < U; ++k) acc += (double)v[k];
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// One warp task: up to 32/W rows of one bin, W lanes per row segment.
template <int PH, int W, int U>
__device__ __forceinline__ double warp_task(const IterArgs& a, int start, int count, int lane,
                                            const float* __restrict__ pr_old, const float* __restrict__ con_old,
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
  double sum = group_row_sum<PH, W, U>(b, e, sl, a.radj, con_old);
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

// One phase of one iteration. Persistent CTAs of 256 threads: long-row chunks
// first (CTA each), then the warp tasks, heaviest bins first.
template <int PH>
__global__ void __launch_bounds__(THREADS) k_phase(IterArgs a, const float* __restrict__ pr_old,
                                                   const float* __restrict__ con_old, float* __restrict__ pr_new,
                                                   float* __restrict__ con_new) {
  __shared__ double s_red[THREADS / 32];
  __shared__ int s_last;
  if (a.st->done) return;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const Phase& P = a.ph[PH];
  double my_diff = 0;

  for (int ci = blockIdx.x; ci < P.n_chunks; ci += gridDim.x) {
    const int4 c = P.chunks[ci];
    double acc = 0;
    {
      int idx[CIPT];
#pragma unroll
      for (int k = 0; k < CIPT; ++k) {
        const int e = c.y + tid + k * THREADS;
        idx[k] = e < c.z ? ld_src<PH>(a.radj + e) : -1;
      }
      float v[CIPT];
#pragma unroll
      for (int k = 0; k < CIPT; ++k) v[k] = idx[k] >= 0 ? __ldg(con_old + idx[k]) : 0.0f;
#pragma unroll
      for (int k = 0; k < CIPT; ++k) acc += (double)v[k];
    }
    const double tot = block_sum<THREADS>(acc, s_red);
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

  const int warps_total = gridDim.x * (THREADS / 32);
  for (int t = blockIdx.x * (THREADS / 32) + (tid >> 5); t < P.n_tasks; t += warps_total) {
    const int4 task = P.tasks[t];  // {W, start, count, -}
    switch (task.x) {
      case 32: my_diff += warp_task<PH, 32, 8>(a, task.y, task.z, lane, pr_old, con_old, pr_new, con_new); break;
      case 8: my_diff += warp_task<PH, 8, 4>(a, task.y, task.z, lane, pr_old, con_old, pr_new, con_new); break;
      case 4: my_diff += warp_task<PH, 4, 4>(a, task.y, task.z, lane, pr_old, con_old, pr_new, con_new); break;
      default: my_diff += warp_task<PH, 1, 4>(a, task.y, task.z, lane, pr_old, con_old, pr_new, con_new); break;
    }
  }

  const double bd = block_sum<THREADS>(my_diff, s_red);
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
    for (int i = (a.two_phase ? 0 : (int)gridDim.x) + tid; i < 2 * (int)gridDim.x; i += THREADS) p += dp[i];
    const double total = block_sum<THREADS>(p, s_red);
    if (tid == 0) {
      const double all = total + *(volatile double*)&a.st->extra;
      const int it = a.st->iter + 1;
      a.st->iter = it;
      a.st->diff = all;
      a.st->done = (all > a.beta && it < a.max_iter) ? 0 : 1;
      a.st->ticket = 0;
      a.st->extra = 0.0;
    }
  }
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
__global__ void k_deg_keys(int V, const int32_t* __restrict__ off, int32_t* __restrict__ key, int32_t* __restrict__ id) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    key[v] = -(off[v + 1] - off[v]);
    id[v] = v;
  }
}

__global__ void k_relabel_rows(int V, const int32_t* __restrict__ inv, const int32_t* __restrict__ skey,
                               const int32_t* __restrict__ roff, int32_t* __restrict__ new_id, int32_t* __restrict__ od,
                               int32_t* __restrict__ indeg) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V; k += gridDim.x * blockDim.x) {
    const int v = inv[k];
    new_id[v] = k;
    od[k] = -skey[k];
    indeg[k] = roff[v + 1] - roff[v];
  }
}

// new row k <- old row inv[k], ids mapped; rows above 1024 in-edges are left to
// k_relabel_adj_big (a whole CTA per row) so one warp never walks a hub alone.
__global__ void k_relabel_adj(int V, const int32_t* __restrict__ inv, const int32_t* __restrict__ new_id,
                              const int32_t* __restrict__ roff, const int32_t* __restrict__ radj,
                              const int32_t* __restrict__ roffp, int32_t* __restrict__ radjp, int32_t* big,
                              int* nbig) {
  const int lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < V; k += (gridDim.x * blockDim.x) >> 5) {
    const int v = inv[k];
    const int b = roff[v], n = roff[v + 1] - b, d = roffp[k];
    if (n > 1024) {
      if (lane == 0) big[atomicAdd(nbig, 1)] = k;
      continue;
    }
    for (int j = lane; j < n; j += 32) radjp[d + j] = new_id[radj[b + j]];
  }
}

__global__ void k_relabel_adj_big(const int32_t* __restrict__ inv, const int32_t* __restrict__ new_id,
                                  const int32_t* __restrict__ roff, const int32_t* __restrict__ radj,
                                  const int32_t* __restrict__ roffp, int32_t* __restrict__ radjp,
                                  const int32_t* __restrict__ big, const int* __restrict__ nbig) {
  for (int i = blockIdx.x; i < *nbig; i += gridDim.x) {
    const int k = big[i], v = inv[k];
    const int b = roff[v], n = roff[v + 1] - b, d = roffp[k];
    for (int j = threadIdx.x; j < n; j += blockDim.x) radjp[d + j] = new_id[radj[b + j]];
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

// Relabel vertices by out-degree on the device: new_id, od, and the reverse CSR in
// new ids with every row sorted.
static int relabel(sp_graph* g, PrPlan* p) {
  const int V = g->V;
  cudaStream_t s = g->stream;
  SP_TRY(p->new_id.alloc(V));
  SP_TRY(p->od.alloc(V));
  SP_TRY(p->roffp.alloc(V + 1));
  SP_TRY(p->radjp.alloc(g->E));
  SP_TRY(p->outbuf.alloc(V));
  dbuf<int32_t> key, id, skey, inv, indeg, big, tmp;
  dbuf<int> nbig;
  SP_TRY(key.alloc(V));
  SP_TRY(id.alloc(V));
  SP_TRY(skey.alloc(V));
  SP_TRY(inv.alloc(V));
  SP_TRY(indeg.alloc(V + 1));
  SP_TRY(big.alloc(V));
  SP_TRY(nbig.alloc(1));
  const int grid = num_sms() * 8;
  pr::k_deg_keys<<<grid, 256, 0, s>>>(V, g->off.p, key.p, id.p);
  SP_CHECK_LAUNCH();
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, skey.p, id.p, inv.p, V, 0, 32, s);
  dbuf<unsigned char> temp;
  SP_TRY(temp.alloc(tb));
  cub::DeviceRadixSort::SortPairs(temp.p, tb, key.p, skey.p, id.p, inv.p, V, 0, 32, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemsetAsync(indeg.p + V, 0, sizeof(int32_t), s));
  pr::k_relabel_rows<<<grid, 256, 0, s>>>(V, inv.p, skey.p, g->roff.p, p->new_id.p, p->od.p, indeg.p);
  SP_CHECK_LAUNCH();
  size_t sb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, sb, indeg.p, p->roffp.p, V + 1, s);
  SP_TRY(temp.alloc(sb));
  cub::DeviceScan::ExclusiveSum(temp.p, sb, indeg.p, p->roffp.p, V + 1, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemsetAsync(nbig.p, 0, sizeof(int), s));
  SP_TRY(tmp.alloc(g->E));
  pr::k_relabel_adj<<<grid, 256, 0, s>>>(V, inv.p, p->new_id.p, g->roff.p, g->radj.p, p->roffp.p, tmp.p, big.p, nbig.p);
  SP_CHECK_LAUNCH();
  pr::k_relabel_adj_big<<<num_sms() * 2, 256, 0, s>>>(inv.p, p->new_id.p, g->roff.p, g->radj.p, p->roffp.p, tmp.p,
                                                       big.p, nbig.p);
  SP_CHECK_LAUNCH();
  size_t xb = 0;
  cub::DeviceSegmentedSort::SortKeys(nullptr, xb, tmp.p, p->radjp.p, (int)g->E, V, p->roffp.p, p->roffp.p + 1, s);
  SP_TRY(temp.alloc(xb));
  cub::DeviceSegmentedSort::SortKeys(temp.p, xb, tmp.p, p->radjp.p, (int)g->E, V, p->roffp.p, p->roffp.p + 1, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  return SP_OK;
}

// Bins of one phase: rows whose segment in this phase is non-empty, by its length.
static void bin_phase(const std::vector<int32_t>& seg_b, const std::vector<int32_t>& seg_e,
                      const std::vector<char>& is_long, std::vector<int32_t>& rows, std::vector<int4>& tasks) {
  const int V = (int)seg_b.size();
  std::vector<int32_t> bin[4];  // W = 32, 8, 4, 1
  for (int r = 0; r < V; ++r) {
    if (is_long[r]) continue;
    const int d = seg_e[r] - seg_b[r];
    if (d <= 0) continue;
    if (d > pr::BIN_T8) bin[0].push_back(r);
    else if (d > pr::BIN_T4) bin[1].push_back(r);
    else if (d > pr::BIN_T1) bin[2].push_back(r);
    else bin[3].push_back(r);
  }
  const int widths[4] = {32, 8, 4, 1};
  rows.clear();
  tasks.clear();
  for (int k = 0; k < 4; ++k) {
    const int per = 32 / widths[k];
    const int base = (int)rows.size();
    rows.insert(rows.end(), bin[k].begin(), bin[k].end());
    for (int i = 0; i < (int)bin[k].size(); i += per)
      tasks.push_back(make_int4(widths[k], base + i, std::min(per, (int)bin[k].size() - i), 0));
  }
}

static int build_pr_plan(sp_graph* g, int hot) {
  if (g->pr && g->pr->hot == hot) return SP_OK;
  SP_TRY(ensure_reverse(g));
  const int V = g->V;
  PrPlan* p = g->pr;
  if (!p) {
    p = new PrPlan();
    int st = relabel(g, p);
    if (st) {
      free_pr_plan(p);
      return st;
    }
    g->pr = p;
  }
  cudaStream_t s = g->stream;
  SP_TRY(p->hot_end.alloc(V));
  pr::k_hot_end<<<num_sms() * 8, 256, 0, s>>>(V, p->roffp.p, p->radjp.p, hot, p->hot_end.p);
  SP_CHECK_LAUNCH();
  std::vector<int32_t> roff(V + 1), hend(V);
  SP_CHECK_CUDA(cudaMemcpyAsync(roff.data(), p->roffp.p, sizeof(int32_t) * (V + 1), cudaMemcpyDeviceToHost, s));
  SP_CHECK_CUDA(cudaMemcpyAsync(hend.data(), p->hot_end.p, sizeof(int32_t) * V, cudaMemcpyDeviceToHost, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  // long rows: chunks in both phases, slots contiguous per row
  std::vector<char> is_long(V, 0);
  std::vector<int4> chunks[2];
  std::vector<int32_t> clong[2];
  std::vector<int2> longs;
  std::vector<int32_t> zrows;
  int slots = 0;
  for (int r = 0; r < V; ++r) {
    const int d = roff[r + 1] - roff[r];
    if (d == 0) {
      zrows.push_back(r);
      continue;
    }
    if (d <= pr::LONG_DEG) continue;
    is_long[r] = 1;
    const int first = slots, li = (int)longs.size();
    const int seg[3] = {roff[r], hend[r], roff[r + 1]};
    for (int ph = 0; ph < 2; ++ph)
      for (int e = seg[ph]; e < seg[ph + 1]; e += pr::CHUNK) {
        chunks[ph].push_back(make_int4(r, e, std::min(e + pr::CHUNK, seg[ph + 1]), slots++));
        clong[ph].push_back(li);
      }
    longs.push_back(make_int2(first, slots - first));
  }
  std::vector<int32_t> rows[2];
  std::vector<int4> tasks[2];
  {
    std::vector<int32_t> b0(V), e0(V), b1(V), e1(V);
    for (int r = 0; r < V; ++r) {
      b0[r] = roff[r];
      e0[r] = hend[r];
      b1[r] = hend[r];
      e1[r] = roff[r + 1];
    }
    bin_phase(b0, e0, is_long, rows[0], tasks[0]);
    bin_phase(b1, e1, is_long, rows[1], tasks[1]);
  }
  const int max_grid = num_sms() * 32;
  for (int ph = 0; ph < 2; ++ph) {
    p->n_tasks[ph] = (int)tasks[ph].size();
    p->n_chunks[ph] = (int)chunks[ph].size();
    SP_TRY(p->rows[ph].alloc(std::max<size_t>(1, rows[ph].size())));
    SP_TRY(p->tasks[ph].alloc(std::max(1, p->n_tasks[ph])));
    SP_TRY(p->chunks[ph].alloc(std::max(1, p->n_chunks[ph])));
    SP_TRY(p->chunk_long[ph].alloc(std::max(1, p->n_chunks[ph])));
    if (!rows[ph].empty())
      SP_CHECK_CUDA(cudaMemcpyAsync(p->rows[ph].p, rows[ph].data(), 4 * rows[ph].size(), cudaMemcpyHostToDevice, s));
    if (p->n_tasks[ph])
      SP_CHECK_CUDA(cudaMemcpyAsync(p->tasks[ph].p, tasks[ph].data(), sizeof(int4) * p->n_tasks[ph], cudaMemcpyHostToDevice, s));
    if (p->n_chunks[ph]) {
      SP_CHECK_CUDA(cudaMemcpyAsync(p->chunks[ph].p, chunks[ph].data(), sizeof(int4) * p->n_chunks[ph], cudaMemcpyHostToDevice, s));
      SP_CHECK_CUDA(cudaMemcpyAsync(p->chunk_long[ph].p, clong[ph].data(), 4 * p->n_chunks[ph], cudaMemcpyHostToDevice, s));
    }
  }
  p->n_long = (int)longs.size();
  p->n_zero = (int)zrows.size();
  SP_TRY(p->longs.alloc(std::max(1, p->n_long)));
  SP_TRY(p->long_ctr.alloc(std::max(1, p->n_long)));
  SP_TRY(p->chunk_part.alloc(std::max(1, slots)));
  SP_TRY(p->zrows.alloc(std::max(1, p->n_zero)));
  SP_TRY(p->part.alloc(V));
  SP_TRY(p->diff_part.alloc(2 * max_grid));
  SP_TRY(p->state.alloc(1));
  for (int i = 0; i < 2; ++i) SP_TRY(p->prb[i].alloc(V));
  for (int i = 0; i < 2; ++i) SP_TRY(p->con[i].alloc(V));
  if (p->n_long)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->longs.p, longs.data(), sizeof(int2) * p->n_long, cudaMemcpyHostToDevice, s));
  if (p->n_zero)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->zrows.p, zrows.data(), 4 * p->n_zero, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->long_ctr.p, 0, sizeof(unsigned int) * std::max(1, p->n_long), s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  if (p->exec) {
    cudaGraphExecDestroy(p->exec);
    p->exec = nullptr;
  }
  p->hot = hot;
  return SP_OK;
}

static int pr_tuned(sp_graph* g, float beta, float delta, int32_t maxIter, float* out, int32_t* iters,
                    double* fdiff) {
  const int hot = std::max(0, std::min(g->pr_hot >= 0 ? g->pr_hot : pr::HOT_DEFAULT, pr::HOT_MAX));
  SP_TRY(build_pr_plan(g, hot));
  PrPlan* p = g->pr;
  cudaStream_t s = g->stream;
  const int V = g->V;
  const int n_iter = std::max(1, (int)maxIter);
  pr::IterArgs a;
  a.roff = p->roffp.p;
  a.radj = p->radjp.p;
  a.hot_end = p->hot_end.p;
  a.od = p->od.p;
  a.longs = p->longs.p;
  a.long_ctr = p->long_ctr.p;
  a.chunk_part = p->chunk_part.p;
  a.part = p->part.p;
  a.diff_part = p->diff_part.p;
  a.st = p->state.p;
  for (int ph = 0; ph < 2; ++ph) {
    a.ph[ph].rows = p->rows[ph].p;
    a.ph[ph].tasks = p->tasks[ph].p;
    a.ph[ph].chunks = p->chunks[ph].p;
    a.ph[ph].chunk_long = p->chunk_long[ph].p;
    a.ph[ph].n_tasks = p->n_tasks[ph];
    a.ph[ph].n_chunks = p->n_chunks[ph];
  }
  a.delta = delta;
  a.base = (1.0f - delta) / (float)V;
  a.beta = (double)beta;
  a.max_iter = n_iter;
  a.two_phase = (p->n_tasks[0] || p->n_chunks[0]) ? 1 : 0;
  int per_sm = 0;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr::k_phase<1>, pr::THREADS, 0));
  const int grid = std::max(1, std::min(num_sms() * 32, num_sms() * std::max(1, per_sm)));

  pr::k_init<<<num_sms() * 4, 256, 0, s>>>(V, p->od.p, p->prb[0].p, p->con[0].p, p->state.p);
  SP_CHECK_LAUNCH();
  if (!(p->exec && p->exec_iters == n_iter && p->exec_beta == beta && p->exec_delta == delta && p->exec_stream == s)) {
    if (p->exec) {
      cudaGraphExecDestroy(p->exec);
      p->exec = nullptr;
    }
    cudaGraph_t graph;
    SP_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < n_iter; ++k) {
      const int c = k & 1, n = c ^ 1;
      if (k < 2 && p->n_zero)
        pr::k_zero_rows<<<num_sms() * 2, 256, 0, s>>>(a, p->zrows.p, p->n_zero, p->prb[c].p, p->prb[n].p, p->con[n].p);
      if (a.two_phase)
        pr::k_phase<0><<<grid, pr::THREADS, 0, s>>>(a, p->prb[c].p, p->con[c].p, p->prb[n].p, p->con[n].p);
      pr::k_phase<1><<<grid, pr::THREADS, 0, s>>>(a, p->prb[c].p, p->con[c].p, p->prb[n].p, p->con[n].p);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
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
    p->exec_stream = s;
  }
  SP_CHECK_CUDA(cudaGraphLaunch(p->exec, s));
  g_launches.fetch_add((unsigned long long)n_iter * ((p->n_tasks[0] || p->n_chunks[0]) ? 2 : 1) +
                       (p->n_zero ? std::min(2, n_iter) : 0));
  pr::State hs;
  SP_TRY(copy_out(&hs, p->state.p, sizeof(hs), s));
  if (out) {
    pr::k_unpermute<<<num_sms() * 4, 256, 0, s>>>(V, p->new_id.p, p->prb[hs.iter & 1].p, p->outbuf.p);
    SP_CHECK_LAUNCH();
    SP_TRY(copy_out(out, p->outbuf.p, sizeof(float) * V, s));
  }
  if (iters) *iters = hs.iter;
  if (fdiff) *fdiff = hs.diff;
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
