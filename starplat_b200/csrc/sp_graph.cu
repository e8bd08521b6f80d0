// Device mirror of the reference CSR container (graphcode/graph.hpp:31-57) and
// library-level C-ABI plumbing (errors, launch counter, streams).
#include <cub/cub.cuh>

#include <cstdarg>
#include <cstring>
#include <mutex>

#include "sp_internal.cuh"

namespace sp {

std::atomic<unsigned long long> g_launches{0};
static thread_local char t_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
}

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return SP_OK;
  SP_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  return SP_OK;
}

// ---------------------------------------------------------------- reverse CSR on device
__global__ void k_count_in(const int32_t* __restrict__ adj, int64_t E, int32_t* __restrict__ cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[adj[e]], 1);
}

__global__ void k_scatter_rev(const int32_t* __restrict__ off, const int32_t* __restrict__ adj, int32_t V,
                              int32_t* __restrict__ cursor, int32_t* __restrict__ radj) {
  // one warp per source vertex
  int lane = threadIdx.x & 31;
  for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; u < V;
       u += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    for (int e = off[u] + lane; e < off[u + 1]; e += 32) {
      int v = adj[e];
      int p = atomicAdd(&cursor[v], 1);
      radj[p] = (int32_t)u;
    }
  }
}

__global__ void k_cmp(const int32_t* __restrict__ a, const int32_t* __restrict__ b, int64_t n,
                      int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (a[i] != b[i]) {
      *bad = 1;
      return;
    }
}

// One warp per vertex: offsets monotone within [0, E], ids in [0, V), adjacency strictly increasing.
__global__ void k_validate_csr(const int32_t* __restrict__ off, const int32_t* __restrict__ adj, int32_t V,
                               int64_t E, int* __restrict__ bad, int32_t* __restrict__ maxdeg) {
  const int lane = threadIdx.x & 31;
  for (int64_t v = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; v < V;
       v += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    int a = off[v], b = off[v + 1];
    if (a > b || a < 0 || b > E) {
      if (lane == 0) atomicOr(bad, 1);
      continue;
    }
    if (lane == 0) atomicMax(maxdeg, b - a);
    int flags = 0;
    for (int e = a + lane; e < b; e += 32) {
      int x = adj[e];
      if (x < 0 || x >= V) flags |= 2;
      if (e + 1 < b && adj[e + 1] <= x) flags |= 4;  // duplicate or unsorted adjacency
    }
    flags = __reduce_or_sync(0xffffffffu, flags);
    if (lane == 0 && flags) atomicOr(bad, flags);
  }
}

int ensure_reverse(sp_graph* g) {
  if (g->has_rev) return SP_OK;
  cudaStream_t s = g->stream;
  SP_TRY(g->roff.alloc(g->V + 1));
  SP_TRY(g->radj.alloc(g->E));
  dbuf<int32_t> cnt, cursor, tmp;
  SP_TRY(cnt.alloc(g->V + 1));
  SP_TRY(cursor.alloc(g->V + 1));
  SP_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (g->V + 1), s));
  int grid = num_sms() * 8;
  k_count_in<<<grid, 256, 0, s>>>(g->adj.p, g->E, cnt.p);
  SP_CHECK_LAUNCH();
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, g->roff.p, g->V + 1, s);
  dbuf<unsigned char> temp;
  SP_TRY(temp.alloc(tb));
  cub::DeviceScan::ExclusiveSum(temp.p, tb, cnt.p, g->roff.p, g->V + 1, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemcpyAsync(cursor.p, g->roff.p, sizeof(int32_t) * g->V, cudaMemcpyDeviceToDevice, s));
  k_scatter_rev<<<grid, 256, 0, s>>>(g->off.p, g->adj.p, g->V, cursor.p, g->radj.p);
  SP_CHECK_LAUNCH();
  // sort each reverse segment (graph.hpp:825-832 sorts srcList per vertex)
  SP_TRY(tmp.alloc(g->E));
  size_t sb = 0;
  cub::DeviceSegmentedSort::SortKeys(nullptr, sb, g->radj.p, tmp.p, (int)g->E, g->V, g->roff.p, g->roff.p + 1, s);
  dbuf<unsigned char> stemp;
  SP_TRY(stemp.alloc(sb));
  cub::DeviceSegmentedSort::SortKeys(stemp.p, sb, g->radj.p, tmp.p, (int)g->E, g->V, g->roff.p, g->roff.p + 1, s);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemcpyAsync(g->radj.p, tmp.p, sizeof(int32_t) * g->E, cudaMemcpyDeviceToDevice, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  g->has_rev = true;
  return SP_OK;
}

int ensure_symmetry(sp_graph* g) {
  if (g->symmetric >= 0) return SP_OK;
  SP_TRY(ensure_reverse(g));
  cudaStream_t s = g->stream;
  dbuf<int> bad;
  SP_TRY(bad.alloc(1));
  SP_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  int grid = num_sms() * 4;
  k_cmp<<<grid, 256, 0, s>>>(g->off.p, g->roff.p, (int64_t)g->V + 1, bad.p);
  SP_CHECK_LAUNCH();
  k_cmp<<<grid, 256, 0, s>>>(g->adj.p, g->radj.p, g->E, bad.p);
  SP_CHECK_LAUNCH();
  int h = 0;
  SP_TRY(copy_out(&h, bad.p, sizeof(int), s));
  g->symmetric = h ? 0 : 1;
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" {

int sp_version(void) { return 10000; }

const char* sp_last_error(void) { return t_err; }

unsigned long long sp_launch_count(void) { return g_launches.load(); }

int sp_graph_create(int32_t V, int64_t E, const int32_t* indexofNodes, const int32_t* edgeList,
                    const int32_t* edgeLen, const int32_t* rev_indexofNodes, const int32_t* srcList,
                    uint32_t flags, sp_graph_h* out) {
  if (!out) {
    set_error("sp_graph_create: out is NULL");
    return SP_ERR_INVALID;
  }
  *out = nullptr;
  if (V <= 0 || E < 0 || E >= (int64_t)INT32_MAX || !indexofNodes || (E > 0 && !edgeList)) {
    set_error("sp_graph_create: invalid sizes or NULL CSR (V=%d E=%lld)", V, (long long)E);
    return SP_ERR_INVALID;
  }
  if ((rev_indexofNodes == nullptr) != (srcList == nullptr)) {
    set_error("sp_graph_create: give both rev_indexofNodes and srcList, or neither");
    return SP_ERR_INVALID;
  }
  const cudaMemcpyKind kind = (flags & SP_GRAPH_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault;
  sp_graph* g = new sp_graph();
  cudaGetDevice(&g->device);
  g->V = V;
  g->E = E;
  auto fail = [&](int st) {
    sp_graph_free(g);
    return st;
  };
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete g;
    set_error("sp_graph_create: cudaStreamCreate failed");
    return SP_ERR_CUDA;
  }
  g->own_stream = true;
  int st;
  if ((st = g->off.alloc(V + 1)) || (st = g->adj.alloc(E))) return fail(st);
  if (cudaMemcpyAsync(g->off.p, indexofNodes, sizeof(int32_t) * (V + 1), kind, g->stream) != cudaSuccess ||
      (E > 0 && cudaMemcpyAsync(g->adj.p, edgeList, sizeof(int32_t) * E, kind, g->stream) != cudaSuccess)) {
    set_error("sp_graph_create: copy of CSR failed");
    return fail(SP_ERR_CUDA);
  }
  if (edgeLen) {
    if ((st = g->w.alloc(E))) return fail(st);
    if (E > 0 && cudaMemcpyAsync(g->w.p, edgeLen, sizeof(int32_t) * E, kind, g->stream) != cudaSuccess) {
      set_error("sp_graph_create: copy of edgeLen failed");
      return fail(SP_ERR_CUDA);
    }
    g->has_w = true;
  }
  // validate: offsets monotone within [0,E], ids in range, adjacency strictly sorted
  {
    dbuf<int> bad;
    dbuf<int32_t> md;
    if ((st = bad.alloc(2)) || (st = md.alloc(1))) return fail(st);
    cudaMemsetAsync(bad.p, 0, sizeof(int) * 2, g->stream);
    cudaMemsetAsync(md.p, 0, sizeof(int32_t), g->stream);
    k_validate_csr<<<num_sms() * 16, 256, 0, g->stream>>>(g->off.p, g->adj.p, V, E, bad.p, md.p);
    g_launches++;
    int h[2] = {0, 0};
    int32_t hm = 0;
    if (copy_out(h, bad.p, sizeof(int), g->stream) || copy_out(&hm, md.p, sizeof(int32_t), g->stream)) return fail(SP_ERR_CUDA);
    int32_t last = 0, first = -1;
    cudaMemcpy(&last, g->off.p + V, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaMemcpy(&first, g->off.p, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (h[0] || last != E || first != 0) {
      set_error("sp_graph_create: malformed CSR (flags=%d, indexofNodes[0]=%d, indexofNodes[V]=%d, E=%lld)", h[0],
                first, last, (long long)E);
      return fail(SP_ERR_INVALID);
    }
    g->max_out_deg = hm;
  }
  if (rev_indexofNodes) {
    if ((st = g->roff.alloc(V + 1)) || (st = g->radj.alloc(E))) return fail(st);
    if (cudaMemcpyAsync(g->roff.p, rev_indexofNodes, sizeof(int32_t) * (V + 1), kind, g->stream) != cudaSuccess ||
        (E > 0 && cudaMemcpyAsync(g->radj.p, srcList, sizeof(int32_t) * E, kind, g->stream) != cudaSuccess)) {
      set_error("sp_graph_create: copy of reverse CSR failed");
      return fail(SP_ERR_CUDA);
    }
    dbuf<int> bad;
    dbuf<int32_t> md;
    if ((st = bad.alloc(1)) || (st = md.alloc(1))) return fail(st);
    cudaMemsetAsync(bad.p, 0, sizeof(int), g->stream);
    k_validate_csr<<<num_sms() * 16, 256, 0, g->stream>>>(g->roff.p, g->radj.p, V, E, bad.p, md.p);
    g_launches++;
    int h = 0;
    int32_t last = -1, first = -1;
    if (copy_out(&h, bad.p, sizeof(int), g->stream)) return fail(SP_ERR_CUDA);
    cudaMemcpy(&last, g->roff.p + V, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaMemcpy(&first, g->roff.p, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (h || last != E || first != 0) {
      set_error("sp_graph_create: malformed reverse CSR (flags=%d)", h);
      return fail(SP_ERR_INVALID);
    }
    g->has_rev = true;
  }
  if (cudaStreamSynchronize(g->stream) != cudaSuccess) {
    set_error("sp_graph_create: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(SP_ERR_CUDA);
  }
  *out = g;
  return SP_OK;
}

int sp_graph_free(sp_graph_h g) {
  if (!g) return SP_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  free_pr_plan(g->pr);
  free_tc_plan(g->tc);
  free_sssp_plan(g->sssp);
  free_bc_plan(g->bc);
  free_lv_plan(g->lv);
  g->off.release();
  g->adj.release();
  g->w.release();
  g->roff.release();
  g->radj.release();
  if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return SP_OK;
}

int sp_graph_set_stream(sp_graph_h g, void* cuda_stream) {
  if (!g) {
    set_error("sp_graph_set_stream: NULL graph");
    return SP_ERR_INVALID;
  }
  cudaStreamSynchronize(g->stream);
  if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
  g->own_stream = false;
  g->stream = (cudaStream_t)cuda_stream;
  if (!cuda_stream) {
    cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    g->own_stream = true;
  }
  return SP_OK;
}

int sp_tune_set(sp_graph_h g, const char* key, int64_t value) {
  if (!g || !key) {
    set_error("sp_tune_set: NULL argument");
    return SP_ERR_INVALID;
  }
  if (!strcmp(key, "pr.hot")) {
    if (value < 0 || value > (1 << 22)) {
      set_error("sp_tune_set: pr.hot must be in [0, 4194304]");
      return SP_ERR_INVALID;
    }
    g->pr_hot = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.delta")) {
    if (value < 0) {
      set_error("sp_tune_set: sssp.delta must be >= 0");
      return SP_ERR_INVALID;
    }
    g->sssp_delta = value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.ctas_per_sm")) {
    if (value < 0 || value > 8) {
      set_error("sp_tune_set: sssp.ctas_per_sm must be in [0, 8]");
      return SP_ERR_INVALID;
    }
    g->sssp_ctas_per_sm = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.batch")) {
    if (value < 0 || value > 64) {
      set_error("sp_tune_set: bc.batch must be in [0, 64]");
      return SP_ERR_INVALID;
    }
    g->bc_batch = (int32_t)value;
    return SP_OK;
  }
  set_error("sp_tune_set: unknown key '%s'", key);
  return SP_ERR_INVALID;
}

int sp_tune_get(sp_graph_h g, const char* key, int64_t* value) {
  if (!g || !key || !value) {
    set_error("sp_tune_get: NULL argument");
    return SP_ERR_INVALID;
  }
  if (!strcmp(key, "pr.hot")) {
    *value = g->pr_hot >= 0 ? g->pr_hot : 0;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.delta")) {
    *value = g->sssp_delta;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.ctas_per_sm")) {
    *value = g->sssp_ctas_per_sm;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_delta")) {
    *value = g->sssp_last_delta;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_ctas")) {
    *value = g->sssp_last_ctas;
    return SP_OK;
  }
  if (!strcmp(key, "bc.batch")) {
    *value = g->bc_batch > 0 ? g->bc_batch : 64;
    return SP_OK;
  }
  set_error("sp_tune_get: unknown key '%s'", key);
  return SP_ERR_INVALID;
}

int sp_graph_info(sp_graph_h g, int32_t* V, int64_t* E, int32_t* symmetric) {
  if (!g) {
    set_error("sp_graph_info: NULL graph");
    return SP_ERR_INVALID;
  }
  if (V) *V = g->V;
  if (E) *E = g->E;
  if (symmetric) {
    SP_TRY(ensure_symmetry(g));
    *symmetric = g->symmetric;
  }
  return SP_OK;
}

}  // extern "C"
