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

// ---------------------------------------------------------------- device block cache
namespace {
struct Block {
  void* p;
  size_t bytes;
  int device;
};
struct BlockCache {
  std::mutex mu;
  std::vector<Block> blocks;
  size_t cached[64] = {};  // bytes held per device
  size_t cap[64] = {};     // at most min(1/8 of the device's memory, 4 GiB) is held
};
// Never destroyed: buffers in static objects may be released during exit.
BlockCache& cache() {
  static BlockCache* c = new BlockCache();
  return *c;
}

// Frees the cached blocks of one device (all devices when dev < 0); returns the bytes.
size_t drain(int dev) {
  BlockCache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  int cur = 0;
  cudaGetDevice(&cur);
  size_t freed = 0;
  for (size_t i = 0; i < c.blocks.size();) {
    const Block b = c.blocks[i];
    if (dev >= 0 && b.device != dev) {
      ++i;
      continue;
    }
    if (b.device != cur) cudaSetDevice(b.device);
    cudaFree(b.p);
    if (b.device != cur) cudaSetDevice(cur);
    c.cached[b.device] -= b.bytes;
    freed += b.bytes;
    c.blocks[i] = c.blocks.back();
    c.blocks.pop_back();
  }
  return freed;
}
}  // namespace

int dev_alloc(void** p, size_t bytes, size_t* got, int* dev) {
  int d = 0;
  cudaGetDevice(&d);
  BlockCache& c = cache();
  {
    // best fit among this device's blocks no larger than twice the request (+1 MiB)
    std::lock_guard<std::mutex> lk(c.mu);
    int best = -1;
    for (int i = 0; i < (int)c.blocks.size(); ++i) {
      const Block& b = c.blocks[i];
      if (b.device == d && b.bytes >= bytes && b.bytes <= 2 * bytes + (1u << 20) &&
          (best < 0 || b.bytes < c.blocks[best].bytes))
        best = i;
    }
    if (best >= 0) {
      const Block b = c.blocks[best];
      c.blocks[best] = c.blocks.back();
      c.blocks.pop_back();
      c.cached[d] -= b.bytes;
      *p = b.p;
      *got = b.bytes;
      *dev = d;
      return SP_OK;
    }
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    drain(d);
    e = cudaMalloc(p, bytes);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    set_error("cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SP_ERR_OOM : SP_ERR_CUDA;
  }
  *got = bytes;
  *dev = d;
  return SP_OK;
}

void dev_free(void* p, size_t bytes, int dev) {
  int cur = 0;
  cudaGetDevice(&cur);
  BlockCache& c = cache();
  if (dev != cur || dev < 0 || dev >= 64) {
    cudaFree(p);
    return;
  }
  // the same ordering cudaFree gives: work still using the block finishes first
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaFree(p);
    return;
  }
  std::lock_guard<std::mutex> lk(c.mu);
  if (!c.cap[dev]) {
    size_t fr = 0, tot = 0;
    // other allocators in the process (torch's) cannot reclaim what this cache holds
    c.cap[dev] = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? std::min(tot / 8, (size_t)4 << 30) : 0;
  }
  if (c.cached[dev] + bytes > c.cap[dev]) {
    cudaFree(p);
    return;
  }
  c.blocks.push_back({p, bytes, dev});
  c.cached[dev] += bytes;
}

// ---------------------------------------------------------------- reverse CSR on device
// Row of every CSR entry, edge-parallel in tiles of EDGE_TILE entries (coalesced writes;
// hub rows spread over many blocks).
__global__ void k_row_of(int32_t V, int64_t E, const int32_t* __restrict__ off, int32_t* __restrict__ row) {
  __shared__ int s_v[2];
  for (long long t0 = (long long)blockIdx.x * EDGE_TILE; t0 < E; t0 += (long long)gridDim.x * EDGE_TILE) {
    const long long t1 = t0 + EDGE_TILE < E ? t0 + EDGE_TILE : E;
    if (threadIdx.x < 2) s_v[threadIdx.x] = edge_source(off, 0, V, threadIdx.x == 0 ? t0 : t1 - 1);
    __syncthreads();
    const int vlo = s_v[0], vhi = s_v[1];
    for (long long e = t0 + threadIdx.x; e < t1; e += blockDim.x) row[e] = edge_source(off, vlo, vhi + 1, e);
    __syncthreads();
  }
}

// off[v] = first index whose sorted key is >= v, for v = 0..V.
__global__ void k_offsets_of_sorted(int32_t V, int64_t E, const int32_t* __restrict__ keys, int32_t* __restrict__ off) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= V; v += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = E;
    while (lo < hi) {
      const int64_t m = (lo + hi) >> 1;
      if (keys[m] < v) lo = m + 1; else hi = m;
    }
    off[v] = (int32_t)lo;
  }
}

// edgeMap: reverse entry i (row r, source u) -> index of r in u's forward row.
__global__ void k_emap(int32_t V, int64_t E, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                       const int32_t* __restrict__ rrow, const int32_t* __restrict__ radj, int32_t* __restrict__ emap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = rrow[i], u = radj[i];
    int lo = off[u], hi = off[u + 1];
    while (lo < hi) {
      const int m = (lo + hi) >> 1;
      if (adj[m] < r) lo = m + 1; else hi = m;
    }
    emap[i] = lo;
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

// CSR check in two coalesced passes (no warp ever walks a hub row alone).
// res[0] = flags: 1 offsets not monotone within [0, E] (or off[0] != 0, off[V] != E),
// 2 an id outside [0, V), 4 a row not strictly increasing (unsorted or duplicate);
// res[1] = maximum row length.
// Row pass: offsets, row lengths, and a bit at the first edge of every non-empty row.
__global__ void k_val_rows(const int32_t* __restrict__ off, int32_t V, int64_t E, uint32_t* __restrict__ starts,
                           int* __restrict__ res) {
  int flags = 0, md = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
    const int a = off[v], b = off[v + 1];
    if (a > b || a < 0 || b > E) {
      flags |= 1;
      continue;
    }
    md = max(md, b - a);
    if (a < b) atomicOr(&starts[a >> 5], 1u << (a & 31));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || off[V] != E)) flags |= 1;
  flags = __reduce_or_sync(0xffffffffu, flags);
  md = __reduce_max_sync(0xffffffffu, md);
  if ((threadIdx.x & 31) == 0) {
    if (flags) atomicOr(&res[0], flags);
    atomicMax(&res[1], md);
  }
}

// Edge pass: ids in range; a step down (adj[e+1] <= adj[e]) is allowed only where
// e+1 starts a row.
__global__ void k_val_edges(const int32_t* __restrict__ adj, int32_t V, int64_t E,
                            const uint32_t* __restrict__ starts, int* __restrict__ res) {
  int flags = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const int x = adj[e];
    if (x < 0 || x >= V) flags |= 2;
    if (e + 1 < E && adj[e + 1] <= x && !((starts[(e + 1) >> 5] >> ((e + 1) & 31)) & 1u)) flags |= 4;
  }
  flags = __reduce_or_sync(0xffffffffu, flags);
  if ((threadIdx.x & 31) == 0 && flags) atomicOr(&res[0], flags);
}

// The same edge pass over a 16-byte aligned adj, four entries per load and two loads
// per thread in flight; entry e + 4 (the next quad's first) closes each quad's check.
// The at most three entries past the last full quad are checked by one thread.
__global__ void k_val_edges_q(const int32_t* __restrict__ adj, int32_t V, int64_t E,
                              const uint32_t* __restrict__ starts, int* __restrict__ res) {
  int flags = 0;
  const int64_t nq = E / 4;
  const int4* q = reinterpret_cast<const int4*>(adj);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  auto quad = [&](const int4 x, int64_t e) {
    const int v[4] = {x.x, x.y, x.z, x.w};
    const uint32_t sw = starts[e >> 5];  // bits of e .. e + 3 (one word: e is a multiple of 4)
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (v[k] < 0 || v[k] >= V) flags |= 2;
#pragma unroll
    for (int k = 1; k < 4; ++k)
      if (v[k] <= v[k - 1] && !((sw >> ((e + k) & 31)) & 1u)) flags |= 4;
    if (e + 4 < E) {
      const int nx = __ldg(adj + e + 4);
      if (nx <= v[3] && !((starts[(e + 4) >> 5] >> ((e + 4) & 31)) & 1u)) flags |= 4;
    }
  };
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i + stride < nq; i += 2 * stride) {
    const int4 a = __ldg(q + i), b = __ldg(q + i + stride);
    quad(a, 4 * i);
    quad(b, 4 * (i + stride));
  }
  if (i < nq) quad(__ldg(q + i), 4 * i);
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int64_t e = nq * 4; e < E; ++e) {
      const int x = adj[e];
      if (x < 0 || x >= V) flags |= 2;
      if (e + 1 < E && adj[e + 1] <= x && !((starts[(e + 1) >> 5] >> ((e + 1) & 31)) & 1u)) flags |= 4;
    }
  flags = __reduce_or_sync(0xffffffffu, flags);
  if ((threadIdx.x & 31) == 0 && flags) atomicOr(&res[0], flags);
}

// Checks a CSR on the device; res (2 ints, device) receives the flags and the maximum
// row length. starts must hold (E + 31) / 32 words.
static int validate_csr(const int32_t* off, const int32_t* adj, int32_t V, int64_t E, uint32_t* starts, int* res,
                        cudaStream_t s) {
  SP_CHECK_CUDA(cudaMemsetAsync(starts, 0, sizeof(uint32_t) * (size_t)((E + 31) / 32 + 1), s));
  SP_CHECK_CUDA(cudaMemsetAsync(res, 0, 2 * sizeof(int), s));
  k_val_rows<<<num_sms() * 8, 256, 0, s>>>(off, V, E, starts, res);
  SP_CHECK_LAUNCH();
  if (E > 0) {
    if ((reinterpret_cast<uintptr_t>(adj) & 15) == 0 && E >= 4) {
      k_val_edges_q<<<num_sms() * 8, 256, 0, s>>>(adj, V, E, starts, res);
      SP_CHECK_LAUNCH();
    } else {
      k_val_edges<<<num_sms() * 8, 256, 0, s>>>(adj, V, E, starts, res);
      SP_CHECK_LAUNCH();
    }
  }
  return SP_OK;
}

// Reverse CSR by a stable transpose: (dst, src) of every forward entry, in forward
// order (ascending src), radix-sorted by dst; a stable sort keeps each row's sources
// ascending, as graph.hpp:825-832 sorts srcList per vertex.
int ensure_reverse(sp_graph* g) {
  if (g->has_rev) return SP_OK;
  cudaStream_t s = g->stream;
  const int V = g->V;
  const int64_t E = g->E;
  SP_TRY(g->roff.alloc((size_t)V + 1));
  SP_TRY(g->radj.alloc(E));
  int bits = 1;
  while (bits < 31 && (1 << bits) < V) ++bits;
  size_t t_sort = 0;
  cub::DoubleBuffer<int32_t> kb(nullptr, nullptr), vb(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, t_sort, kb, vb, (int)E, 0, bits, s);
  Arena T;
  dspan<int32_t> keys, keys_alt, src, src_alt;
  dspan<unsigned char> temp;
  T.want(keys, E);
  T.want(keys_alt, E);
  T.want(src, E);
  T.want(src_alt, E);
  T.want(temp, t_sort);
  SP_TRY(T.commit());
  if (E > 0) {
    SP_CHECK_CUDA(cudaMemcpyAsync(keys.p, g->adj.p, 4 * (size_t)E, cudaMemcpyDeviceToDevice, s));
    k_row_of<<<num_sms() * 8, 256, 0, s>>>(V, E, g->off.p, src.p);
    SP_CHECK_LAUNCH();
    cub::DoubleBuffer<int32_t> kd(keys.p, keys_alt.p), vd(src.p, src_alt.p);
    size_t t = temp.n;
    SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, kd, vd, (int)E, 0, bits, s));
    g_launches++;
    SP_CHECK_CUDA(cudaMemcpyAsync(g->radj.p, vd.Current(), 4 * (size_t)E, cudaMemcpyDeviceToDevice, s));
    k_offsets_of_sorted<<<num_sms() * 8, 256, 0, s>>>(V, E, kd.Current(), g->roff.p);
    SP_CHECK_LAUNCH();
  } else {
    SP_CHECK_CUDA(cudaMemsetAsync(g->roff.p, 0, sizeof(int32_t) * ((size_t)V + 1), s));
  }
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  g->has_rev = true;
  return SP_OK;
}

int offsets_of_sorted(int32_t V, int64_t E, const int32_t* keys, int32_t* off, cudaStream_t s) {
  if (E > 0) {
    k_offsets_of_sorted<<<num_sms() * 8, 256, 0, s>>>(V, E, keys, off);
    SP_CHECK_LAUNCH();
  } else {
    SP_CHECK_CUDA(cudaMemsetAsync(off, 0, sizeof(int32_t) * ((size_t)V + 1), s));
  }
  return SP_OK;
}

int ensure_emap(sp_graph* g) {
  if (g->emap.p && g->emap.n >= (size_t)g->E) return SP_OK;
  SP_TRY(ensure_reverse(g));
  cudaStream_t s = g->stream;
  const int64_t E = g->E;
  SP_TRY(g->emap.alloc(E));
  if (E > 0) {
    dbuf<int32_t> rrow;
    SP_TRY(rrow.alloc(E));
    k_row_of<<<num_sms() * 8, 256, 0, s>>>(g->V, E, g->roff.p, rrow.p);
    SP_CHECK_LAUNCH();
    k_emap<<<num_sms() * 8, 256, 0, s>>>(g->V, E, g->off.p, g->adj.p, rrow.p, g->radj.p, g->emap.p);
    SP_CHECK_LAUNCH();
    SP_CHECK_CUDA(cudaStreamSynchronize(s));
  }
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

// Checks a CSR built inside the library (both directions when present) and records
// the largest out-degree, as sp_graph_create does for a caller's arrays.
int finish_graph(sp_graph* g) {
  const int64_t E = g->E;
  const size_t nw = (size_t)((E + 31) / 32) + 1;
  dbuf<uint32_t> scratch;
  SP_TRY(scratch.alloc(nw + 4));
  int* res = (int*)(scratch.p + nw);
  SP_TRY(validate_csr(g->off.p, g->adj.p, g->V, E, scratch.p, res, g->stream));
  if (g->has_rev) SP_TRY(validate_csr(g->roff.p, g->radj.p, g->V, E, scratch.p, res + 2, g->stream));
  int h[4] = {0, 0, 0, 0};
  SP_TRY(copy_out(h, res, sizeof(h), g->stream));
  if (h[0] || (g->has_rev && h[2])) {
    set_error("internal CSR check failed (flags %d / %d)", h[0], h[2]);
    return SP_ERR_INVALID;
  }
  g->max_out_deg = h[1];
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" {

int sp_version(void) { return 10000; }

const char* sp_last_error(void) { return t_err; }

unsigned long long sp_launch_count(void) { return g_launches.load(); }

int sp_cache_bytes(int64_t* bytes) {
  if (!bytes) {
    set_error("sp_cache_bytes: NULL output");
    return SP_ERR_INVALID;
  }
  int d = 0;
  cudaGetDevice(&d);
  BlockCache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  *bytes = (d >= 0 && d < 64) ? (int64_t)c.cached[d] : 0;
  return SP_OK;
}

int sp_cache_trim(int64_t* bytes_freed) {
  const size_t f = drain(-1);
  if (bytes_freed) *bytes_freed = (int64_t)f;
  return SP_OK;
}

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
  // A blocking stream: ordered with the legacy default stream in both directions, so
  // device inputs written there (and readers of device outputs there) need no extra sync.
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamDefault) != cudaSuccess) {
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
  if (rev_indexofNodes) {
    if ((st = g->roff.alloc(V + 1)) || (st = g->radj.alloc(E))) return fail(st);
    if (cudaMemcpyAsync(g->roff.p, rev_indexofNodes, sizeof(int32_t) * (V + 1), kind, g->stream) != cudaSuccess ||
        (E > 0 && cudaMemcpyAsync(g->radj.p, srcList, sizeof(int32_t) * E, kind, g->stream) != cudaSuccess)) {
      set_error("sp_graph_create: copy of reverse CSR failed");
      return fail(SP_ERR_CUDA);
    }
  }
  // validate both CSRs: offsets monotone from 0 to E, ids in range, rows strictly increasing
  {
    const size_t nw = (size_t)((E + 31) / 32) + 1;
    dbuf<uint32_t> scratch;
    if ((st = scratch.alloc(nw + 4))) return fail(st);
    int* res = (int*)(scratch.p + nw);  // forward {flags, max degree}, reverse {flags, max degree}
    if ((st = validate_csr(g->off.p, g->adj.p, V, E, scratch.p, res, g->stream))) return fail(st);
    if (rev_indexofNodes && (st = validate_csr(g->roff.p, g->radj.p, V, E, scratch.p, res + 2, g->stream)))
      return fail(st);
    int h[4] = {0, 0, 0, 0};
    if (copy_out(h, res, sizeof(h), g->stream)) return fail(SP_ERR_CUDA);
    if (h[0]) {
      set_error("sp_graph_create: malformed CSR (flags=%d: 1 offsets, 2 ids, 4 unsorted or duplicate row)", h[0]);
      return fail(SP_ERR_INVALID);
    }
    if (rev_indexofNodes && h[2]) {
      set_error("sp_graph_create: malformed reverse CSR (flags=%d: 1 offsets, 2 ids, 4 unsorted or duplicate row)",
                h[2]);
      return fail(SP_ERR_INVALID);
    }
    g->max_out_deg = h[1];
    g->has_rev = rev_indexofNodes != nullptr;
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
  free_sssp_part_plan(g->sssp_part);
  g->off.release();
  g->adj.release();
  g->w.release();
  g->roff.release();
  g->radj.release();
  g->emap.release();
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
    cudaStreamCreateWithFlags(&g->stream, cudaStreamDefault);
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
  if (!strcmp(key, "pr.src_hint")) {
    if (value < 0 || value > 2) {
      set_error("sp_tune_set: pr.src_hint must be 0, 1 or 2");
      return SP_ERR_INVALID;
    }
    g->pr_src_hint = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "pr.l1_hot")) {
    if (value < 0 || value > (1 << 22)) {
      set_error("sp_tune_set: pr.l1_hot must be in [0, 4194304]");
      return SP_ERR_INVALID;
    }
    g->pr_l1_hot = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "pr.vec")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: pr.vec must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->pr_vec = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "pr.order")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: pr.order must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->pr_order = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.dir")) {
    if (value < -1 || value > 4) {
      set_error("sp_tune_set: bc.dir must be -1, 0, 1, 2, 3 or 4");
      return SP_ERR_INVALID;
    }
    g->bc_dir = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.pull_alpha")) {
    if (value < 0 || value > 1000000000) {
      set_error("sp_tune_set: bc.pull_alpha must be in [0, 1e9] (thousandths)");
      return SP_ERR_INVALID;
    }
    g->bc_pull_alpha = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.dir_seed")) {
    g->bc_dir_seed = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.trace")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: bc.trace must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->bc_trace = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.epoch")) {
    if (value < -1 || value > 2) {
      set_error("sp_tune_set: sssp.epoch must be -1, 0, 1 or 2");
      return SP_ERR_INVALID;
    }
    g->sssp_epoch = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.epoch_widen")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: sssp.epoch_widen must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->sssp_epoch_widen = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.epoch_seed")) {
    g->sssp_epoch_seed = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.trace")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: sssp.trace must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->sssp_trace = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.batch")) {
    if (value < 0 || value > 1024) {
      set_error("sp_tune_set: sssp.batch must be in [0, 1024]");
      return SP_ERR_INVALID;
    }
    g->sssp_batch = (int32_t)value;
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
  if (!strcmp(key, "sssp.hub_deg") || !strcmp(key, "sssp.hub_chunk")) {
    if (value < 0 || value > (1 << 30)) {
      set_error("sp_tune_set: %s must be in [0, 2^30]", key);
      return SP_ERR_INVALID;
    }
    if (!strcmp(key, "sssp.hub_deg"))
      g->sssp_hub_deg = (int32_t)value;
    else
      g->sssp_hub_chunk = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.repair")) {
    if (value < -1 || value > 1) {
      set_error("sp_tune_set: sssp.repair must be -1, 0 or 1");
      return SP_ERR_INVALID;
    }
    g->sssp_repair = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.filter")) {
    if (value < -1 || value > 1) {
      set_error("sp_tune_set: sssp.filter must be -1, 0 or 1");
      return SP_ERR_INVALID;
    }
    g->sssp_filter = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.local")) {
    if (value < 0 || value > (1 << 16)) {
      set_error("sp_tune_set: sssp.local must be in [0, 65536]");
      return SP_ERR_INVALID;
    }
    g->sssp_local = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.cluster")) {
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8) {
      set_error("sp_tune_set: bc.cluster must be 0, 1, 2, 4 or 8");
      return SP_ERR_INVALID;
    }
    g->bc_cluster = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.hub_deg")) {
    if (value < 0 || value > (1 << 30)) {
      set_error("sp_tune_set: bc.hub_deg must be in [0, 2^30]");
      return SP_ERR_INVALID;
    }
    g->bc_hub_deg = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "bc.hub_chunk")) {
    if (value < 0 || value > (1 << 20)) {
      set_error("sp_tune_set: bc.hub_chunk must be in [0, 2^20]");
      return SP_ERR_INVALID;
    }
    g->bc_hub_chunk = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "tc.cta_warps")) {
    if (value != 0 && value != 2 && value != 4 && value != 8 && value != 16) {
      set_error("sp_tune_set: tc.cta_warps must be 0, 2, 4, 8 or 16");
      return SP_ERR_INVALID;
    }
    g->tc_cta_warps = (int32_t)value;
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
  if (!strcmp(key, "tc.unroll")) {
    if (value != 1 && value != 2 && value != 4) {
      set_error("sp_tune_set: tc.unroll must be 1, 2 or 4");
      return SP_ERR_INVALID;
    }
    g->tc_unroll = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "lv.cta_slots")) {
    if (value != 1024 && value != 2048 && value != 4096 && value != 8192 && value != 16384) {
      set_error("sp_tune_set: lv.cta_slots must be 1024, 2048, 4096, 8192 or 16384");
      return SP_ERR_INVALID;
    }
    g->lv_cta_slots = (int32_t)value;
    return SP_OK;
  }
  if (!strcmp(key, "lv.trace")) {
    if (value != 0 && value != 1) {
      set_error("sp_tune_set: lv.trace must be 0 or 1");
      return SP_ERR_INVALID;
    }
    g->lv_trace = (int32_t)value;
    return SP_OK;
  }
  {
    static const char* const vkeys[VAR_ALGOS] = {"pr.variant", "tc.variant", "bc.variant", "lv.variant"};
    for (int a = 0; a < VAR_ALGOS; ++a)
      if (!strcmp(key, vkeys[a])) {
        int32_t n = 0;
        sp_variant_count(a, &n);
        if (value < -2 || value >= n) {
          set_error("sp_tune_set: %s must be -2 (defaults), -1 (learned) or a candidate in [0, %d)", key, n);
          return SP_ERR_INVALID;
        }
        g->variant[a] = (int32_t)value;
        return SP_OK;
      }
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
  if (!strcmp(key, "pr.src_hint")) {
    *value = g->pr_src_hint >= 0 ? g->pr_src_hint : pr_src_hint_default();
    return SP_OK;
  }
  if (!strcmp(key, "pr.order")) {
    *value = g->pr_order >= 0 ? g->pr_order : pr_order_default();
    return SP_OK;
  }
  if (!strcmp(key, "pr.l1_hot")) {
    *value = g->pr_l1_hot >= 0 ? g->pr_l1_hot : pr_l1_hot_default();
    return SP_OK;
  }
  if (!strcmp(key, "pr.vec")) {
    *value = g->pr_vec >= 0 ? g->pr_vec : pr_vec_default();
    return SP_OK;
  }
  if (!strcmp(key, "sssp.delta")) {
    *value = g->sssp_delta;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.batch")) {
    *value = g->sssp_batch > 0 ? g->sssp_batch : sssp_batch_default();
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_batch")) {
    *value = g->sssp_last_batch;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.epoch")) {
    *value = g->sssp_epoch;
    return SP_OK;
  }
  if (!strcmp(key, "bc.dir")) {
    *value = g->bc_dir;
    return SP_OK;
  }
  if (!strcmp(key, "bc.pull_alpha")) {
    *value = g->bc_pull_alpha;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_epochs")) {
    *value = g->sssp_last_epochs;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_epolicy")) {
    *value = g->sssp_last_epolicy;
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
  if (!strcmp(key, "sssp.last_local")) {
    *value = g->sssp_last_local;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_relaxed")) {
    *value = g->sssp_last_relaxed;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_incremental")) {
    *value = g->sssp_last_incremental;
    return SP_OK;
  }
  if (!strcmp(key, "tc.last_incremental")) {
    *value = g->tc_last_incremental;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.hub_deg")) {
    *value = g->sssp_hub_deg > 0 ? g->sssp_hub_deg : sssp_hub_deg_default();
    return SP_OK;
  }
  if (!strcmp(key, "sssp.hub_chunk")) {
    *value = g->sssp_hub_chunk > 0 ? g->sssp_hub_chunk : sssp_hub_chunk_default();
    return SP_OK;
  }
  if (!strcmp(key, "sssp.filter")) {
    *value = g->sssp_filter;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.repair")) {
    *value = g->sssp_repair;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.last_marked")) {
    *value = g->sssp_last_marked;
    return SP_OK;
  }
  if (!strcmp(key, "sssp.local")) {
    *value = g->sssp_local >= 0 ? g->sssp_local : sssp_local_default();
    return SP_OK;
  }
  if (!strcmp(key, "bc.cluster")) {
    *value = g->bc_cluster > 0 ? g->bc_cluster : bc_cluster_default();
    return SP_OK;
  }
  if (!strcmp(key, "bc.hub_deg")) {
    *value = g->bc_hub_deg > 0 ? g->bc_hub_deg : bc_hub_deg_default();
    return SP_OK;
  }
  if (!strcmp(key, "bc.hub_chunk")) {
    *value = g->bc_hub_chunk > 0 ? g->bc_hub_chunk : bc_hub_chunk_default();
    return SP_OK;
  }
  if (!strcmp(key, "tc.cta_warps")) {
    *value = g->tc_cta_warps >= 0 ? g->tc_cta_warps : tc_cta_warps_default();
    return SP_OK;
  }
  if (!strcmp(key, "bc.batch")) {
    *value = g->bc_batch > 0 ? g->bc_batch : 64;
    return SP_OK;
  }
  if (!strcmp(key, "tc.unroll")) {
    *value = g->tc_unroll > 0 ? g->tc_unroll : 4;
    return SP_OK;
  }
  if (!strcmp(key, "lv.cta_slots")) {
    *value = g->lv_cta_slots > 0 ? g->lv_cta_slots : 16384;
    return SP_OK;
  }
  if (!strcmp(key, "lv.trace")) {
    *value = g->lv_trace;
    return SP_OK;
  }
  {
    static const char* const vkeys[VAR_ALGOS] = {"pr.", "tc.", "bc.", "lv."};
    for (int a = 0; a < VAR_ALGOS; ++a)
      if (!strncmp(key, vkeys[a], 3)) {
        if (!strcmp(key + 3, "variant")) {
          *value = g->variant[a];
          return SP_OK;
        }
        if (!strcmp(key + 3, "last_variant")) {
          *value = g->last_variant[a];
          return SP_OK;
        }
      }
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
