// PageRank, pull form over the reverse CSR, for sm_100a.
//
// Semantics: DSL staticDSLCodes/PageRankDSLV3:1-25 as emitted by the CUDA generator
// (backend_cuda/dsl_cpp_generator.cpp:1472-1480 reads d_src = srcList, count_outNbrs
// :3113-3121): pr0 = 1/V; pr'[v] = (1-delta)/V + delta * sum_{u->v} pr[u]/outdeg(u);
// diff = sum |pr' - pr|; repeat while diff > beta && iter < maxIter.
//
// Design (one kernel launch per iteration, all iterations in one CUDA graph):
//  * Every iteration writes contrib[v] = pr[v]/outdeg(v) next to pr[v], so the next
//    gather reads one float per in-edge (the same per-edge quotient the reference
//    forms in float).
//  * Load balance by static in-degree bins built once per graph: 1, 4, 8 or 32 lanes
//    per row (in-degree <= 4, <= 16, <= 32, <= 2048) with every load of a row in
//    flight at once, and 2048-edge chunks (one CTA each) above that; the CTA that
//    finishes a hub's last chunk adds the chunk partials in chunk order.
//  * Row sums are FP64 and rounded once to FP32; every sum has a fixed order, so the
//    result is deterministic (no float atomics).
//  * The L1 diff is reduced per CTA and summed in CTA order by the last CTA to
//    finish, which also advances the iteration count and raises the done flag; later
//    launches in the graph see the flag and return at once.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "sp_internal.cuh"

namespace sp {

namespace pr {
constexpr int THREADS = 256;
constexpr int CIPT = 8;                 // loads in flight per thread in chunk sums
constexpr int CHUNK = THREADS * CIPT;   // edges per long-row chunk (one round per CTA)
constexpr int HOT_MAX = 56 * 1024;      // largest shared-memory contrib table
constexpr int HOT_DEFAULT = 0;          // measured best on R-MAT 22 (L1/L2 gathers beat shared-memory ones)
constexpr int LONG_DEG = 2048;          // rows above this are chunked (CHUNK-edge pieces)
// degree-bin upper bounds for 1, 4, 8 and 32 lanes per row
constexpr int BIN_T1 = 4, BIN_T4 = 16, BIN_T8 = 32;

struct State {
  int iter;
  int done;
  unsigned int ticket;
  int pad;
  double diff;
};
}  // namespace pr

struct PrPlan {
  int n_chunks = 0, n_long = 0, n_tasks = 0;
  dbuf<int32_t> new_id;   // vertex -> rank by out-degree (descending, stable)
  dbuf<int32_t> od;       // out-degree, in relabelled order
  dbuf<int32_t> roffp, radjp;  // reverse CSR in relabelled ids (per-row order kept)
  dbuf<float> outbuf;     // result in original vertex order
  dbuf<int32_t> rows;     // row ids grouped by in-degree bin
  dbuf<int4> tasks;       // warp tasks {W, start, count, 0}
  dbuf<int4> chunks;      // [n_chunks] {row, e_begin, e_end, long index}
  dbuf<int2> longs;       // [n_long] {first chunk, chunk count}
  dbuf<unsigned int> long_ctr;
  dbuf<double> chunk_part;
  dbuf<double> diff_part;
  dbuf<float> prb[2], con[2];
  dbuf<pr::State> state;
  dbuf<int32_t> outdeg;   // plain variant
  cudaGraphExec_t exec = nullptr;
  int exec_iters = 0;
  float exec_beta = -1, exec_delta = -1;
  cudaStream_t exec_stream = nullptr;
  int exec_hot = -1;
};

void free_pr_plan(PrPlan* p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  p->chunks.release();
  p->rows.release();
  p->new_id.release();
  p->od.release();
  p->roffp.release();
  p->radjp.release();
  p->outbuf.release();
  p->tasks.release();
  p->longs.release();
  p->long_ctr.release();
  p->chunk_part.release();
  p->diff_part.release();
  for (int i = 0; i < 2; ++i) {
    p->prb[i].release();
    p->con[i].release();
  }
  p->state.release();
  p->outdeg.release();
  delete p;
}

namespace pr {

struct IterArgs {
  const int32_t* __restrict__ roff;
  const int32_t* __restrict__ radj;
  const int32_t* __restrict__ od;    // out-degree per (relabelled) row
  const int4* __restrict__ chunks;
  const int2* __restrict__ longs;
  const int32_t* __restrict__ rows;   // binned row ids
  const int4* __restrict__ tasks;     // warp tasks {W, start, count, 0}
  unsigned int* long_ctr;
  double* chunk_part;
  double* diff_part;
  State* st;
  int V;
  int n_chunks;
  int n_tasks;
  int hot;       // multiple of 4, <= V: contrib[0..hot) is read from shared memory
  float base;   // (1 - delta) / V, in float as the DSL computes it
  float delta;
  double beta;
  int max_iter;
};

__device__ __forceinline__ double finalize_row(const IterArgs& a, int r, double sum,
                                               const float* __restrict__ pr_old, float* __restrict__ pr_new,
                                               float* __restrict__ con_new) {
  float s = (float)sum;
  float np = __fadd_rn(a.base, __fmul_rn(a.delta, s));
  float po = pr_old[r];
  pr_new[r] = np;
  int od = a.od[r];
  con_new[r] = od > 0 ? __fdiv_rn(np, (float)od) : 0.0f;
  return fabs((double)np - (double)po);
}

// contrib of relabelled vertex u: the first `hot` ids (highest out-degree, so the
// most gathered) come from the shared-memory copy, the rest from global memory.
__device__ __forceinline__ float gather(const float* __restrict__ con, const float* s_hot, int hot, int u) {
  return u < hot ? s_hot[u] : __ldg(con + u);
}

// Sum of con[radj[i]] for i in [b, e) by a group of W lanes (sl = lane within the
// group), U loads in flight per lane per round, reduced with a fixed xor tree.
template <int W, int U>
__device__ __forceinline__ double group_row_sum(int b, int e, int sl, const int32_t* __restrict__ radj,
                                                const float* __restrict__ con, const float* s_hot, int hot) {
  double acc = 0;
  for (int base = b; base < e; base += W * U) {
    int idx[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      int i = base + sl + W * k;
      idx[k] = i < e ? __ldg(radj + i) : -1;
    }
    float v[U];
#pragma unroll
    for (int k = 0; k < U; ++k) v[k] = idx[k] >= 0 ? gather(con, s_hot, hot, idx[k]) : 0.0f;
#pragma unroll
    for (int k = 0; k < U; ++k) acc += (double)v[k];
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

template <int W, int U>
__device__ __forceinline__ double warp_task(const IterArgs& a, int start, int count, int lane, const float* s_hot,
                                            const float* __restrict__ pr_old, const float* __restrict__ con_old,
                                            float* __restrict__ pr_new, float* __restrict__ con_new) {
  const int g = lane / W, sl = lane % W;
  int r = -1, b = 0, e = 0;
  if (g < count) {
    r = a.rows[start + g];
    b = a.roff[r];
    e = a.roff[r + 1];
  }
  double sum = group_row_sum<W, U>(b, e, sl, a.radj, con_old, s_hot, a.hot);
  if (r >= 0 && sl == 0) return finalize_row(a, r, sum, pr_old, pr_new, con_new);
  return 0.0;
}

// One iteration. Persistent CTAs of 256 threads:
//  phase 1: in-degree > 2048: 2048-edge chunks, one CTA each (CTA-strided); the CTA
//           that adds a row's last chunk partial finalizes the row (arrival counter);
//  phase 2: warp tasks (warp-strided), heaviest bins first: up to 32/W rows of one
//           degree bin, W lanes per row, all of a row's loads in flight at once
//           (W = 32 for in-degree 33..2048, 8 for 17..32, 4 for 5..16, 1 for 0..4).
// Row sums are FP64 with a fixed order per row, so results are deterministic.
__global__ void __launch_bounds__(THREADS) k_iter(IterArgs a, const float* __restrict__ pr_old,
                                                  const float* __restrict__ con_old, float* __restrict__ pr_new,
                                                  float* __restrict__ con_new) {
  extern __shared__ float4 s_dyn[];
  float* s_hot = reinterpret_cast<float*>(s_dyn);
  __shared__ double s_red[THREADS / 32];
  __shared__ int s_last;
  if (a.st->done) return;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  double my_diff = 0;
  {
    const float4* src = reinterpret_cast<const float4*>(con_old);
    for (int i = tid; i < a.hot / 4; i += THREADS) s_dyn[i] = __ldg(src + i);
    __syncthreads();
  }

  for (int ci = blockIdx.x; ci < a.n_chunks; ci += gridDim.x) {
    const int4 c = a.chunks[ci];
    double acc = 0;
    {
      int idx[CIPT];
#pragma unroll
      for (int k = 0; k < CIPT; ++k) {
        int e = c.y + tid + k * THREADS;
        idx[k] = e < c.z ? __ldg(a.radj + e) : -1;
      }
      float v[CIPT];
#pragma unroll
      for (int k = 0; k < CIPT; ++k) v[k] = idx[k] >= 0 ? gather(con_old, s_hot, a.hot, idx[k]) : 0.0f;
#pragma unroll
      for (int k = 0; k < CIPT; ++k) acc += (double)v[k];
    }
    double tot = block_sum<THREADS>(acc, s_red);
    if (tid == 0) {
      a.chunk_part[ci] = tot;
      __threadfence();
      const int2 L = a.longs[c.w];
      unsigned int old = atomicAdd(&a.long_ctr[c.w], 1u);
      s_last = (old == (unsigned)(L.y - 1));
    }
    __syncthreads();
    if (s_last && tid == 0) {
      __threadfence();
      const int2 L = a.longs[c.w];
      double sum = 0;
      const volatile double* cp = a.chunk_part;
      for (int k = 0; k < L.y; ++k) sum += cp[L.x + k];
      my_diff += finalize_row(a, c.x, sum, pr_old, pr_new, con_new);
      a.long_ctr[c.w] = 0;
    }
    __syncthreads();
  }

  const int warps_total = gridDim.x * (THREADS / 32);
  for (int t = blockIdx.x * (THREADS / 32) + (tid >> 5); t < a.n_tasks; t += warps_total) {
    const int4 task = a.tasks[t];  // {W, start, count, -}
    switch (task.x) {
      case 32: my_diff += warp_task<32, 8>(a, task.y, task.z, lane, s_hot, pr_old, con_old, pr_new, con_new); break;
      case 8: my_diff += warp_task<8, 4>(a, task.y, task.z, lane, s_hot, pr_old, con_old, pr_new, con_new); break;
      case 4: my_diff += warp_task<4, 4>(a, task.y, task.z, lane, s_hot, pr_old, con_old, pr_new, con_new); break;
      default: my_diff += warp_task<1, 4>(a, task.y, task.z, lane, s_hot, pr_old, con_old, pr_new, con_new); break;
    }
  }

  // per-CTA diff partial, then the last CTA reduces them in CTA order
  double bd = block_sum<THREADS>(my_diff, s_red);
  if (tid == 0) {
    a.diff_part[blockIdx.x] = bd;
    __threadfence();
    unsigned int t = atomicAdd(&a.st->ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const volatile double* dp = a.diff_part;
    double p = 0;
    for (int i = tid; i < (int)gridDim.x; i += THREADS) p += dp[i];
    double total = block_sum<THREADS>(p, s_red);
    if (tid == 0) {
      int it = a.st->iter + 1;
      a.st->iter = it;
      a.st->diff = total;
      a.st->done = (total > a.beta && it < a.max_iter) ? 0 : 1;
      a.st->ticket = 0;
    }
  }
}

// ---- relabelling by out-degree (descending): the most gathered contrib values
// share cache lines and stay resident in L1
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
    int v = inv[k];
    new_id[v] = k;
    od[k] = -skey[k];
    indeg[k] = roff[v + 1] - roff[v];
  }
}

__global__ void k_relabel_adj(int V, const int32_t* __restrict__ inv, const int32_t* __restrict__ new_id,
                              const int32_t* __restrict__ roff, const int32_t* __restrict__ radj,
                              const int32_t* __restrict__ roffp, int32_t* __restrict__ radjp) {
  const int lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < V; k += (gridDim.x * blockDim.x) >> 5) {
    const int v = inv[k];
    const int b = roff[v], n = roff[v + 1] - b, d = roffp[k];
    for (int j = lane; j < n; j += 32) radjp[d + j] = new_id[radj[b + j]];
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
    int od = odeg[v];
    con[v] = od > 0 ? __fdiv_rn(p0, (float)od) : 0.0f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->done = 0;
    st->ticket = 0;
    st->diff = 0;
  }
}

// ---- plain variant: the generated CUDA form (one thread per vertex, serial gather
// of pr[u]/outdeg(u), atomic float diff; backend_cuda/dsl_cpp_generator.cpp:1682-1761)
__global__ void k_plain_iter(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ roff,
                             const int32_t* __restrict__ radj, const float* __restrict__ pr,
                             float* __restrict__ prn, float base, float delta, float* diff) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  float sum = 0.0f;
  for (int e = roff[v]; e < roff[v + 1]; ++e) {
    int u = radj[e];
    sum = sum + pr[u] / (float)(off[u + 1] - off[u]);
  }
  float np = base + delta * sum;
  atomicAdd(diff, fabsf(np - pr[v]));
  prn[v] = np;
}

__global__ void k_plain_init(int V, float* pr) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) pr[v] = 1.0f / (float)V;
}

}  // namespace pr

// Relabel vertices by out-degree on the device: new_id, od, and the reverse CSR
// in new ids (rows in new order, each row's in-neighbours in their original order).
static int relabel(sp_graph* g, PrPlan* p) {
  const int V = g->V;
  cudaStream_t s = g->stream;
  SP_TRY(p->new_id.alloc(V));
  SP_TRY(p->od.alloc(V));
  SP_TRY(p->roffp.alloc(V + 1));
  SP_TRY(p->radjp.alloc(g->E));
  SP_TRY(p->outbuf.alloc(V));
  dbuf<int32_t> key, id, skey, inv, indeg;
  SP_TRY(key.alloc(V));
  SP_TRY(id.alloc(V));
  SP_TRY(skey.alloc(V));
  SP_TRY(inv.alloc(V));
  SP_TRY(indeg.alloc(V + 1));
  const int grid = num_sms() * 8;
  pr::k_deg_keys<<<grid, 256, 0, s>>>(V, g->off.p, key.p, id.p);
  SP_CHECK_LAUNCH();
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, skey.p, id.p, inv.p, V, 0, 32, s);
  dbuf<unsigned char> tmp;
  SP_TRY(tmp.alloc(tb));
  cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, skey.p, id.p, inv.p, V, 0, 32, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemsetAsync(indeg.p + V, 0, sizeof(int32_t), s));
  pr::k_relabel_rows<<<grid, 256, 0, s>>>(V, inv.p, skey.p, g->roff.p, p->new_id.p, p->od.p, indeg.p);
  SP_CHECK_LAUNCH();
  size_t sb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, sb, indeg.p, p->roffp.p, V + 1, s);
  dbuf<unsigned char> stmp;
  SP_TRY(stmp.alloc(sb));
  cub::DeviceScan::ExclusiveSum(stmp.p, sb, indeg.p, p->roffp.p, V + 1, s);
  SP_CHECK_LAUNCH();
  pr::k_relabel_adj<<<grid, 256, 0, s>>>(V, inv.p, p->new_id.p, g->roff.p, g->radj.p, p->roffp.p, p->radjp.p);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  return SP_OK;
}

static int build_pr_plan(sp_graph* g) {
  if (g->pr) return SP_OK;
  SP_TRY(ensure_reverse(g));
  const int V = g->V;
  PrPlan* p = new PrPlan();
  {
    int st = relabel(g, p);
    if (st) {
      free_pr_plan(p);
      return st;
    }
  }
  std::vector<int32_t> roff(V + 1);
  SP_CHECK_CUDA(cudaMemcpyAsync(roff.data(), p->roffp.p, sizeof(int32_t) * (V + 1), cudaMemcpyDeviceToHost, g->stream));
  SP_CHECK_CUDA(cudaStreamSynchronize(g->stream));
  std::vector<int4> chunks;
  std::vector<int2> longs;
  std::vector<int32_t> bin[4];  // W = 32, 8, 4, 1
  for (int r = 0; r < V; ++r) {
    int deg = roff[r + 1] - roff[r];
    if (deg > pr::LONG_DEG) {
      int first = (int)chunks.size();
      for (int e = roff[r]; e < roff[r + 1]; e += pr::CHUNK)
        chunks.push_back(make_int4(r, e, std::min(e + pr::CHUNK, roff[r + 1]), (int)longs.size()));
      longs.push_back(make_int2(first, (int)chunks.size() - first));
    } else if (deg > pr::BIN_T8) {
      bin[0].push_back(r);
    } else if (deg > pr::BIN_T4) {
      bin[1].push_back(r);
    } else if (deg > pr::BIN_T1) {
      bin[2].push_back(r);
    } else {
      bin[3].push_back(r);
    }
  }
  // warp tasks, heaviest bin first; rows concatenated in the same order
  const int widths[4] = {32, 8, 4, 1};
  std::vector<int32_t> rows;
  std::vector<int4> tasks;
  rows.reserve(V);
  for (int k = 0; k < 4; ++k) {
    const int per = 32 / widths[k];
    const int base = (int)rows.size();
    rows.insert(rows.end(), bin[k].begin(), bin[k].end());
    for (int i = 0; i < (int)bin[k].size(); i += per)
      tasks.push_back(make_int4(widths[k], base + i, std::min(per, (int)bin[k].size() - i), 0));
  }
  p->n_chunks = (int)chunks.size();
  p->n_long = (int)longs.size();
  p->n_tasks = (int)tasks.size();
  int st;
  auto fail = [&](int s) {
    free_pr_plan(p);
    return s;
  };
  const int max_grid = num_sms() * 32;
  if ((st = p->chunks.alloc(std::max(1, p->n_chunks))) || (st = p->longs.alloc(std::max(1, p->n_long))) ||
      (st = p->long_ctr.alloc(std::max(1, p->n_long))) || (st = p->chunk_part.alloc(std::max(1, p->n_chunks))) ||
      (st = p->diff_part.alloc(max_grid)) || (st = p->state.alloc(1)) ||
      (st = p->rows.alloc(std::max<size_t>(1, rows.size()))) || (st = p->tasks.alloc(std::max(1, p->n_tasks))))
    return fail(st);
  for (int i = 0; i < 2; ++i)
    if ((st = p->prb[i].alloc(V)) || (st = p->con[i].alloc(V))) return fail(st);
  cudaStream_t s = g->stream;
  if (p->n_chunks)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->chunks.p, chunks.data(), sizeof(int4) * p->n_chunks, cudaMemcpyHostToDevice, s));
  if (p->n_long)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->longs.p, longs.data(), sizeof(int2) * p->n_long, cudaMemcpyHostToDevice, s));
  if (!rows.empty())
    SP_CHECK_CUDA(cudaMemcpyAsync(p->rows.p, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice, s));
  if (p->n_tasks)
    SP_CHECK_CUDA(cudaMemcpyAsync(p->tasks.p, tasks.data(), sizeof(int4) * p->n_tasks, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->long_ctr.p, 0, sizeof(unsigned int) * std::max(1, p->n_long), s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  g->pr = p;
  return SP_OK;
}

static int pr_tuned(sp_graph* g, float beta, float delta, int32_t maxIter, float* out, int32_t* iters,
                    double* fdiff) {
  SP_TRY(build_pr_plan(g));
  PrPlan* p = g->pr;
  cudaStream_t s = g->stream;
  const int V = g->V;
  const int n_iter = std::max(1, (int)maxIter);
  pr::IterArgs a;
  a.roff = p->roffp.p;
  a.radj = p->radjp.p;
  a.od = p->od.p;
  a.chunks = p->chunks.p;
  a.longs = p->longs.p;
  a.long_ctr = p->long_ctr.p;
  a.chunk_part = p->chunk_part.p;
  a.diff_part = p->diff_part.p;
  a.st = p->state.p;
  a.rows = p->rows.p;
  a.tasks = p->tasks.p;
  a.V = V;
  a.n_chunks = p->n_chunks;
  a.n_tasks = p->n_tasks;
  a.delta = delta;
  a.base = (1.0f - delta) / (float)V;
  a.beta = (double)beta;
  a.max_iter = n_iter;
  int hot = std::min(g->pr_hot >= 0 ? g->pr_hot : pr::HOT_DEFAULT, pr::HOT_MAX);
  hot = std::min(hot, V) & ~3;
  a.hot = hot;
  const size_t dyn = std::max<size_t>(16, sizeof(float) * (size_t)hot);
  SP_CHECK_CUDA(cudaFuncSetAttribute(pr::k_iter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  int per_sm = 0;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr::k_iter, pr::THREADS, dyn));
  const int grid = std::max(1, std::min(num_sms() * 32, num_sms() * std::max(1, per_sm)));

  pr::k_init<<<num_sms() * 4, 256, 0, s>>>(V, p->od.p, p->prb[0].p, p->con[0].p, p->state.p);
  SP_CHECK_LAUNCH();
  if (!(p->exec && p->exec_iters == n_iter && p->exec_beta == beta && p->exec_delta == delta && p->exec_stream == s &&
        p->exec_hot == hot)) {
    if (p->exec) {
      cudaGraphExecDestroy(p->exec);
      p->exec = nullptr;
    }
    cudaGraph_t graph;
    SP_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < n_iter; ++k) {
      int c = k & 1, n = c ^ 1;
      pr::k_iter<<<grid, pr::THREADS, dyn, s>>>(a, p->prb[c].p, p->con[c].p, p->prb[n].p, p->con[n].p);
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
    p->exec_hot = hot;
  }
  SP_CHECK_CUDA(cudaGraphLaunch(p->exec, s));
  g_launches.fetch_add(n_iter);
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
  SP_TRY(build_pr_plan(g));
  PrPlan* p = g->pr;
  cudaStream_t s = g->stream;
  const int V = g->V;
  dbuf<float> d_diff;
  SP_TRY(d_diff.alloc(1));
  const int tb = 512;  // the generator's launch shape (backend_cuda/dsl_cpp_generator.cpp:56-77)
  const int nb = (V + tb - 1) / tb;
  pr::k_plain_init<<<nb, tb, 0, s>>>(V, p->prb[0].p);
  SP_CHECK_LAUNCH();
  const float base = (1.0f - delta) / (float)V;
  int it = 0;
  float diff = 0;
  int cur = 0;
  do {
    SP_CHECK_CUDA(cudaMemsetAsync(d_diff.p, 0, sizeof(float), s));
    pr::k_plain_iter<<<nb, tb, 0, s>>>(V, g->off.p, g->roff.p, g->radj.p, p->prb[cur].p, p->prb[cur ^ 1].p, base,
                                        delta, d_diff.p);
    SP_CHECK_LAUNCH();
    SP_TRY(copy_out(&diff, d_diff.p, sizeof(float), s));
    cur ^= 1;
    ++it;
  } while (diff > beta && it < maxIter);
  if (out) SP_TRY(copy_out(out, p->prb[cur].p, sizeof(float) * V, s));
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
