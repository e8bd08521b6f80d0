// Text edge-list ingestion: the reference's graph::parseGraph (graph.hpp:464-512
// parseEdges, :720-865 parseEdgesContent) rebuilt for a GPU host.
//
// Reference semantics kept:
//  * one edge per line "src dst weight"; a line that is empty or does not start with
//    a digit is skipped (comments, headers, blank lines) (:471-474);
//  * fields are whitespace separated integers as std::stringstream reads them: an
//    optional sign, digits up to the first other character ("3.7" reads 3); a
//    malformed weight reads 0; one out of int32 range saturates (:478-490);
//  * the vertex count is the largest id + 1 (nodesTotal starts at 0) (:483-487, :139);
//  * duplicate (src, dst) pairs become one edge whose weight is the sum (:493-506);
//    self-loops are kept;
//  * forward rows sorted by destination, reverse rows sorted by source, and
//    edgeMap[i] = forward index of reverse entry i (:725-859).
// Where the reference is undefined this build decides: a line without a weight field
// gets weight 1 (the reference leaves it uninitialised), and a missing, malformed,
// negative or out-of-range source / destination is an error naming the line (the
// reference stores 0 or a negative id and indexes out of its arrays).
//
// B200 design: host threads tokenise disjoint byte ranges of the file (the only
// per-byte work), the triples go to the device once, and everything else runs
// there: a radix sort of (src << 32 | dst) keys with their weights, a
// reduce-by-key for the duplicate sums, the forward offsets by binary search, and
// the reverse CSR and edgeMap by a stable transpose (ensure_reverse). The reference
// spends its time in a std::map insertion per line and an O(indeg^2) edgeMap loop.
#include <cub/cub.cuh>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sp_internal.cuh"

namespace sp {

namespace ingest {

struct Part {
  std::vector<int32_t> s, d, w;
  int64_t lines = 0;      // lines that start in this part
  int32_t max_id = 0;
  int64_t err_line = -1;  // line index within the part
  const char* err = nullptr;
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// An integer as stringstream's operator>> reads it: optional sign, then digits up to
// the first non-digit. 0 = ok, 1 = no digits, 2 = out of int32 range (v saturated).
inline int read_int(const char*& p, const char* end, int32_t& v) {
  bool neg = false;
  if (p < end && (*p == '+' || *p == '-')) {
    neg = *p == '-';
    ++p;
  }
  if (p >= end || *p < '0' || *p > '9') return 1;
  long long x = 0;
  bool over = false;
  for (; p < end && *p >= '0' && *p <= '9'; ++p) {
    if (!over) {
      x = x * 10 + (*p - '0');
      if (x > (long long)INT_MAX + 1) over = true;
    }
  }
  if (neg) x = -x;
  if (over || x > INT_MAX || x < INT_MIN) {
    v = neg ? INT_MIN : INT_MAX;
    return 2;
  }
  v = (int32_t)x;
  return 0;
}

// Parses the lines that start in [lo, hi) of buf[0, n).
void parse_part(const char* buf, size_t n, size_t lo, size_t hi, Part& out) {
  size_t pos = lo;
  if (lo > 0) {  // the line containing lo belongs to the previous part
    while (pos < n && buf[pos - 1] != '\n') ++pos;
  }
  out.s.reserve((hi - lo) / 12 + 16);
  out.d.reserve((hi - lo) / 12 + 16);
  out.w.reserve((hi - lo) / 12 + 16);
  while (pos < hi && pos < n) {
    const char* a = buf + pos;
    const char* nl = (const char*)memchr(a, '\n', n - pos);
    const char* b = nl ? nl : buf + n;
    pos = (size_t)(b - buf) + 1;
    const int64_t line = out.lines++;
    if (a == b || *a < '0' || *a > '9') continue;
    const char* p = a;
    int32_t src = 0, dst = 0, w = 1;
    if (read_int(p, b, src) != 0) {
      out.err_line = line;
      out.err = "source id out of int32 range";
      return;
    }
    while (p < b && is_space(*p)) ++p;
    const int rd = read_int(p, b, dst);
    if (rd != 0 || dst < 0) {
      out.err_line = line;
      out.err = rd == 1 ? "missing or malformed destination" : "destination id negative or out of int32 range";
      return;
    }
    while (p < b && is_space(*p)) ++p;
    if (p < b) {
      const int rw = read_int(p, b, w);
      if (rw == 1) w = 0;  // a malformed field reads as 0
    }
    if (src == INT_MAX || dst == INT_MAX) {
      out.err_line = line;
      out.err = "vertex id too large (the vertex count would exceed int32)";
      return;
    }
    out.s.push_back(src);
    out.d.push_back(dst);
    out.w.push_back(w);
    out.max_id = std::max(out.max_id, std::max(src, dst));
  }
}

__global__ void k_pack(int64_t n, const int32_t* __restrict__ s, const int32_t* __restrict__ d,
                       unsigned long long* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = ((unsigned long long)(uint32_t)s[i] << 32) | (uint32_t)d[i];
}

// Forward CSR from the sorted unique keys: adj = low halves; off[v] = first key whose
// source is >= v (binary search, one thread per vertex, v = 0..V).
__global__ void k_forward(int32_t V, int64_t E, const unsigned long long* __restrict__ ukeys,
                          int32_t* __restrict__ off, int32_t* __restrict__ adj) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = tid; e < E; e += stride) adj[e] = (int32_t)(uint32_t)(ukeys[e] & 0xffffffffull);
  for (int64_t v = tid; v <= V; v += stride) {
    int64_t lo = 0, hi = E;
    while (lo < hi) {
      const int64_t m = (lo + hi) >> 1;
      if ((int64_t)(ukeys[m] >> 32) < v) lo = m + 1; else hi = m;
    }
    off[v] = (int32_t)lo;
  }
}

// ---- one batch of edge updates, merged into the sorted CSR (update_graph) ----------
// The current edges are already sorted (src, dst) keys, so the batch is merged in
// instead of sorting everything again. The batch's deletion keys are sorted and made
// unique (udel), each flagged if the CSR holds it, and the flags scanned: xrank[j] is
// the number of held deletion keys below udel[j]. The additions are sorted, duplicates
// summed (uak, uaw), each flagged fresh if it adds an edge (absent from the CSR, or
// deleted by the batch), and the flags scanned into newrank. An edge with key k then
// moves from i to i - xrank[lb(udel, k)] + newrank[lb(uak, k)], and a fresh addition j
// with key q to newrank[j] + (CSR keys below q) - xrank[lb(udel, q)]. A radix sort of
// all keys took 2.5 ms of a 3.5 ms update on undirected R-MAT 20 (31M edges).

__device__ __forceinline__ int lb_u64(const unsigned long long* __restrict__ a, int n, unsigned long long k) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (a[m] < k) lo = m + 1; else hi = m;
  }
  return lo;
}

// First index in the sorted row adj[b .. e) whose entry is >= x.
__device__ __forceinline__ int lb_row(const int32_t* __restrict__ adj, int b, int e, int x) {
  while (b < e) {
    const int m = (b + e) >> 1;
    if (adj[m] < x) b = m + 1; else e = m;
  }
  return b;
}

__device__ __forceinline__ bool held(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                     unsigned long long k) {
  const int a = (int)(k >> 32), b = (int)(k & 0xffffffffull);
  const int e = off[a + 1], p = lb_row(adj, off[a], e, b);
  return p < e && adj[p] == b;
}

__global__ void k_del_held(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                           const unsigned long long* __restrict__ udel, int nud, int32_t* __restrict__ flag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nud; j += gridDim.x * blockDim.x)
    flag[j] = held(off, adj, udel[j]) ? 1 : 0;
}

__global__ void k_add_fresh(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const unsigned long long* __restrict__ uak, int nua,
                            const unsigned long long* __restrict__ udel, int nud, int32_t* __restrict__ flag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nua; j += gridDim.x * blockDim.x) {
    const unsigned long long k = uak[j];
    const int d = lb_u64(udel, nud, k);
    flag[j] = !held(off, adj, k) || (d < nud && udel[d] == k) ? 1 : 0;
  }
}

// The current edges to their new places (tiles of EDGE_TILE entries); a held edge that
// the batch adds again keeps its place and gains the added weight. A sum outside int32
// raises *overflow (the host then rejects the batch and keeps the old CSR).
__global__ void k_merge_edges(int32_t V, long long E, const int32_t* __restrict__ off,
                              const int32_t* __restrict__ adj, const int32_t* __restrict__ w,
                              const unsigned long long* __restrict__ udel, int nud, const int32_t* __restrict__ xrank,
                              const unsigned long long* __restrict__ uak, const int32_t* __restrict__ uaw, int nua,
                              const int32_t* __restrict__ newrank, int32_t* __restrict__ adj2,
                              int32_t* __restrict__ w2, int* __restrict__ overflow) {
  __shared__ int s_v[2];
  for (long long t0 = (long long)blockIdx.x * EDGE_TILE; t0 < E; t0 += (long long)gridDim.x * EDGE_TILE) {
    const long long t1 = t0 + EDGE_TILE < E ? t0 + EDGE_TILE : E;
    if (threadIdx.x < 2) s_v[threadIdx.x] = edge_source(off, 0, V, threadIdx.x == 0 ? t0 : t1 - 1);
    __syncthreads();
    const int vlo = s_v[0], vhi = s_v[1];
    for (long long i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
      const int u = edge_source(off, vlo, vhi + 1, i);
      const int v = adj[i];
      const unsigned long long k = ((unsigned long long)(uint32_t)u << 32) | (uint32_t)v;
      const int j = lb_u64(udel, nud, k);
      if (j < nud && udel[j] == k) continue;  // deleted
      const int l = lb_u64(uak, nua, k);
      const long long pos = i - xrank[j] + newrank[l];
      adj2[pos] = v;
      if (w2) {
        const long long s = (long long)w[i] + (l < nua && uak[l] == k ? uaw[l] : 0);
        if (s > INT_MAX || s < INT_MIN) *overflow = 1;
        w2[pos] = (int32_t)s;
      }
    }
    __syncthreads();  // s_v is rewritten for the next tile
  }
}

__global__ void k_merge_adds(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                             const unsigned long long* __restrict__ uak, const int32_t* __restrict__ uaw, int nua,
                             const int32_t* __restrict__ newrank, const unsigned long long* __restrict__ udel,
                             int nud, const int32_t* __restrict__ xrank, int32_t* __restrict__ adj2,
                             int32_t* __restrict__ w2) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nua; j += gridDim.x * blockDim.x) {
    if (newrank[j + 1] == newrank[j]) continue;  // a held edge: merged in k_merge_edges
    const unsigned long long k = uak[j];
    const int a = (int)(k >> 32), b = (int)(k & 0xffffffffull);
    const int below = lb_row(adj, off[a], off[a + 1], b);  // CSR keys below k
    const long long pos = (long long)newrank[j] + below - xrank[lb_u64(udel, nud, k)];
    adj2[pos] = b;
    if (w2) w2[pos] = uaw[j];
  }
}

__global__ void k_merge_off(int32_t V, const int32_t* __restrict__ off, const unsigned long long* __restrict__ udel,
                            int nud, const int32_t* __restrict__ xrank, const unsigned long long* __restrict__ uak,
                            int nua, const int32_t* __restrict__ newrank, int32_t* __restrict__ off2) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v <= V; v += gridDim.x * blockDim.x) {
    const unsigned long long k = (unsigned long long)(uint32_t)v << 32;
    off2[v] = off[v] - xrank[lb_u64(udel, nud, k)] + newrank[lb_u64(uak, nua, k)];
  }
}

}  // namespace ingest

// The file mapped read-only (no copy of its bytes), unmapped on scope exit.
struct Mapped {
  const char* p = nullptr;
  size_t n = 0;
  ~Mapped() {
    if (p) munmap((void*)p, n);
  }
};

static int load_text(const char* path, int nthreads, sp_graph_h* out) {
  Mapped file;
  {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) {
      set_error("sp_graph_load_text: cannot open %s", path);
      return SP_ERR_INVALID;
    }
    struct stat sb;
    if (fstat(fd, &sb) != 0) {
      close(fd);
      set_error("sp_graph_load_text: cannot stat %s", path);
      return SP_ERR_INVALID;
    }
    if (sb.st_size > 0) {
      void* m = mmap(nullptr, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m == MAP_FAILED) {
        close(fd);
        set_error("sp_graph_load_text: cannot map %s", path);
        return SP_ERR_INVALID;
      }
      madvise(m, (size_t)sb.st_size, MADV_SEQUENTIAL);
      file.p = (const char*)m;
      file.n = (size_t)sb.st_size;
    }
    close(fd);
  }
  const char* buf = file.p;
  const size_t n = file.n;

  int T = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  T = std::max(1, std::min(T, 64));
  if (n < ((size_t)1 << 20)) T = 1;
  std::vector<ingest::Part> parts(T);
  {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
      th.emplace_back(ingest::parse_part, buf, n, n * t / T, n * (t + 1) / T, std::ref(parts[t]));
    for (auto& x : th) x.join();
  }
  int64_t line0 = 0, m = 0;
  int32_t max_id = 0;
  for (int t = 0; t < T; ++t) {
    if (parts[t].err) {
      set_error("sp_graph_load_text: %s:%lld: %s", path, (long long)(line0 + parts[t].err_line + 1), parts[t].err);
      return SP_ERR_INVALID;
    }
    line0 += parts[t].lines;
    m += (int64_t)parts[t].s.size();
    max_id = std::max(max_id, parts[t].max_id);
  }
  if (m > INT_MAX) {
    set_error("sp_graph_load_text: %lld edge lines (int32 edge indices)", (long long)m);
    return SP_ERR_UNSUPPORTED;
  }
  const int32_t V = max_id + 1;
  sp_graph* g = new sp_graph();
  auto fail = [&](int st) {
    sp_graph_free(g);
    return st;
  };
  cudaGetDevice(&g->device);
  g->V = V;
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamDefault) != cudaSuccess) {
    delete g;
    set_error("sp_graph_load_text: cudaStreamCreate failed");
    return SP_ERR_CUDA;
  }
  g->own_stream = true;
  cudaStream_t s = g->stream;
  int st;
  {
    Arena T0;
    dspan<int32_t> ds, dd, dw, dw_alt, uw;
    dspan<unsigned long long> keys, keys_alt, ukeys;
    dspan<int> nrun;
    dspan<unsigned char> temp;
    int bits = 1;
    while (bits < 31 && (1 << bits) < V) ++bits;
    size_t t_sort = 0, t_red = 0;
    cub::DoubleBuffer<unsigned long long> kb(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> vb(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, t_sort, kb, vb, (int)m, 0, 32 + bits, s);
    cub::DeviceReduce::ReduceByKey(nullptr, t_red, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                   (int32_t*)nullptr, (int32_t*)nullptr, (int*)nullptr, cub::Sum(), (int)m, s);
    T0.want(ds, m);
    T0.want(dd, m);
    T0.want(dw, m);
    T0.want(dw_alt, m);
    T0.want(uw, m);
    T0.want(keys, m);
    T0.want(keys_alt, m);
    T0.want(ukeys, m);
    T0.want(nrun, 1);
    T0.want(temp, std::max(t_sort, t_red));
    if ((st = T0.commit())) return fail(st);
    const size_t tb = temp.n;
    if (m > 0) {
      // each thread's triples go to their place in the device arrays
      int64_t at = 0;
      for (int t = 0; t < T; ++t) {
        const size_t k = parts[t].s.size();
        if (!k) continue;
        if (cudaMemcpyAsync(ds.p + at, parts[t].s.data(), 4 * k, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(dd.p + at, parts[t].d.data(), 4 * k, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(dw.p + at, parts[t].w.data(), 4 * k, cudaMemcpyHostToDevice, s) != cudaSuccess) {
          set_error("sp_graph_load_text: copy to the device failed");
          return fail(SP_ERR_CUDA);
        }
        at += (int64_t)k;
      }
      ingest::k_pack<<<num_sms() * 8, 256, 0, s>>>(m, ds.p, dd.p, keys.p);
      g_launches++;
      cub::DoubleBuffer<unsigned long long> kd(keys.p, keys_alt.p);
      cub::DoubleBuffer<int32_t> vd(dw.p, dw_alt.p);
      size_t t = tb;
      if (cub::DeviceRadixSort::SortPairs(temp.p, t, kd, vd, (int)m, 0, 32 + bits, s) != cudaSuccess) return fail(SP_ERR_CUDA);
      t = tb;
      if (cub::DeviceReduce::ReduceByKey(temp.p, t, kd.Current(), ukeys.p, vd.Current(), uw.p, nrun.p, cub::Sum(),
                                         (int)m, s) != cudaSuccess)
        return fail(SP_ERR_CUDA);
      g_launches += 2;
    }
    int E = 0;
    if (m > 0 && (st = copy_out(&E, nrun.p, sizeof(int), s))) return fail(st);
    g->E = E;
    if ((st = g->off.alloc((size_t)V + 1)) || (st = g->adj.alloc(E)) || (st = g->w.alloc(E))) return fail(st);
    if (E > 0) {
      ingest::k_forward<<<num_sms() * 8, 256, 0, s>>>(V, E, ukeys.p, g->off.p, g->adj.p);
      g_launches++;
      if (cudaMemcpyAsync(g->w.p, uw.p, 4 * (size_t)E, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return fail(SP_ERR_CUDA);
    } else if (cudaMemsetAsync(g->off.p, 0, sizeof(int32_t) * ((size_t)V + 1), s) != cudaSuccess) {
      return fail(SP_ERR_CUDA);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("sp_graph_load_text: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(SP_ERR_CUDA);
    }
  }
  g->has_w = true;
  if ((st = ensure_reverse(g))) return fail(st);
  if ((st = finish_graph(g))) return fail(st);
  *out = g;
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_graph_load_text(const char* path, int32_t nthreads, sp_graph_h* out) {
  if (!path || !out) {
    set_error("sp_graph_load_text: NULL argument");
    return SP_ERR_INVALID;
  }
  *out = nullptr;
  return load_text(path, nthreads, out);
}

namespace sp {

// A batch of edge updates applied to the forward CSR on the device: deletions, then
// additions (see sp_graph_update). Everything derived from the old CSR is dropped.
int update_graph(sp_graph* g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                 const int32_t* weight, int64_t* held_adds) {
  const int32_t V = g->V;
  std::vector<unsigned long long> del;
  std::vector<int32_t> as, ad, aw;
  del.reserve(n);
  as.reserve(n);
  ad.reserve(n);
  aw.reserve(n);
  for (int64_t i = 0; i < n; ++i) {
    if (type[i] != 'a' && type[i] != 'd') {
      set_error("sp_graph_update: update %lld has type '%c' (expected 'a' or 'd')", (long long)i, type[i]);
      return SP_ERR_INVALID;
    }
    if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) {
      set_error("sp_graph_update: update %lld names an edge %d -> %d outside [0, %d)", (long long)i, src[i], dst[i],
                V);
      return SP_ERR_INVALID;
    }
    if (type[i] == 'd') {
      del.push_back(((unsigned long long)(uint32_t)src[i] << 32) | (uint32_t)dst[i]);
    } else {
      as.push_back(src[i]);
      ad.push_back(dst[i]);
      aw.push_back(weight ? weight[i] : 1);
    }
  }
  const int64_t E = g->E, na = (int64_t)as.size(), m = E + na, nd = (int64_t)del.size();
  {  // repeated additions of one edge are summed in int32 on the device: reject a sum that wraps
    int64_t mag = 0;
    for (int32_t x : aw) mag += x < 0 ? -(int64_t)x : (int64_t)x;
    if (mag > INT_MAX) {  // rare: check the per-edge sums exactly
      std::vector<std::pair<unsigned long long, int64_t>> kw((size_t)na);
      for (int64_t i = 0; i < na; ++i)
        kw[i] = {((unsigned long long)(uint32_t)as[i] << 32) | (uint32_t)ad[i], (int64_t)aw[i]};
      std::sort(kw.begin(), kw.end());
      for (size_t i = 0; i < kw.size();) {
        size_t j = i;
        int64_t sum = 0;
        for (; j < kw.size() && kw[j].first == kw[i].first; ++j) sum += kw[j].second;
        if (sum > INT_MAX || sum < INT_MIN) {
          set_error("sp_graph_update: the added weights of edge %d -> %d sum to %lld (outside int32)",
                    (int)(kw[i].first >> 32), (int)(kw[i].first & 0xffffffffull), (long long)sum);
          return SP_ERR_INVALID;
        }
        i = j;
      }
    }
  }
  if (m > INT_MAX) {
    set_error("sp_graph_update: %lld edges after the update (int32 edge indices)", (long long)m);
    return SP_ERR_UNSUPPORTED;
  }
  cudaStream_t s = g->stream;
  int bits = 1;  // key bits above 32: ids below V
  while (bits < 31 && (1 << bits) < V) ++bits;
  Arena T0;
  dspan<unsigned long long> dk, dk_alt, udel, ak, ak_alt, uak;
  dspan<int32_t> xflag, xrank, awd, awd_alt, uaw, fresh, newrank, das, dad;
  dspan<int> cnt;
  dspan<unsigned char> temp;
  size_t t_need = 0;
  {
    size_t t = 0;
    cub::DoubleBuffer<unsigned long long> kb(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> vb(nullptr, nullptr);
    cub::DeviceRadixSort::SortKeys(nullptr, t, kb, (int)nd, 0, 32 + bits, s);
    t_need = std::max(t_need, t);
    cub::DeviceSelect::Unique(nullptr, t, (unsigned long long*)nullptr, (unsigned long long*)nullptr, (int*)nullptr,
                              (int)nd, s);
    t_need = std::max(t_need, t);
    cub::DeviceRadixSort::SortPairs(nullptr, t, kb, vb, (int)na, 0, 32 + bits, s);
    t_need = std::max(t_need, t);
    cub::DeviceReduce::ReduceByKey(nullptr, t, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                   (int32_t*)nullptr, (int32_t*)nullptr, (int*)nullptr, cub::Sum(), (int)na, s);
    t_need = std::max(t_need, t);
    cub::DeviceScan::ExclusiveSum(nullptr, t, (int32_t*)nullptr, (int32_t*)nullptr, (int)std::max(nd, na) + 1, s);
    t_need = std::max(t_need, t);
  }
  T0.want(dk, nd);
  T0.want(dk_alt, nd);
  T0.want(udel, nd);
  T0.want(xflag, nd + 1);
  T0.want(xrank, nd + 1);
  T0.want(ak, na);
  T0.want(ak_alt, na);
  T0.want(uak, na);
  T0.want(awd, na);
  T0.want(awd_alt, na);
  T0.want(uaw, na);
  T0.want(fresh, na + 1);
  T0.want(newrank, na + 1);
  T0.want(das, na);
  T0.want(dad, na);
  T0.want(cnt, 3);
  T0.want(temp, std::max<size_t>(t_need, 16));
  SP_TRY(T0.commit());
  SP_CHECK_CUDA(cudaMemsetAsync(xflag.p, 0, sizeof(int32_t) * (nd + 1), s));
  SP_CHECK_CUDA(cudaMemsetAsync(fresh.p, 0, sizeof(int32_t) * (na + 1), s));
  SP_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * 3, s));
  if (nd > 0) {  // deletion keys: sorted, unique
    SP_CHECK_CUDA(cudaMemcpyAsync(dk.p, del.data(), sizeof(unsigned long long) * nd, cudaMemcpyHostToDevice, s));
    cub::DoubleBuffer<unsigned long long> kd(dk.p, dk_alt.p);
    size_t t = temp.n;
    SP_CHECK_CUDA(cub::DeviceRadixSort::SortKeys(temp.p, t, kd, (int)nd, 0, 32 + bits, s));
    t = temp.n;
    SP_CHECK_CUDA(cub::DeviceSelect::Unique(temp.p, t, kd.Current(), udel.p, cnt.p, (int)nd, s));
    g_launches += 2;
  }
  if (na > 0) {  // addition keys: sorted, duplicates summed
    SP_CHECK_CUDA(cudaMemcpyAsync(das.p, as.data(), 4 * (size_t)na, cudaMemcpyHostToDevice, s));
    SP_CHECK_CUDA(cudaMemcpyAsync(dad.p, ad.data(), 4 * (size_t)na, cudaMemcpyHostToDevice, s));
    SP_CHECK_CUDA(cudaMemcpyAsync(awd.p, aw.data(), 4 * (size_t)na, cudaMemcpyHostToDevice, s));
    ingest::k_pack<<<num_sms() * 4, 256, 0, s>>>(na, das.p, dad.p, ak.p);
    SP_CHECK_LAUNCH();
    cub::DoubleBuffer<unsigned long long> kd(ak.p, ak_alt.p);
    cub::DoubleBuffer<int32_t> vd(awd.p, awd_alt.p);
    size_t t = temp.n;
    SP_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, t, kd, vd, (int)na, 0, 32 + bits, s));
    t = temp.n;
    SP_CHECK_CUDA(cub::DeviceReduce::ReduceByKey(temp.p, t, kd.Current(), uak.p, vd.Current(), uaw.p, cnt.p + 1,
                                                 cub::Sum(), (int)na, s));
    g_launches += 2;
  }
  int hc[2] = {0, 0};
  SP_TRY(copy_out(hc, cnt.p, sizeof(hc), s));
  const int nud = hc[0], nua = hc[1];
  if (nud > 0) {
    ingest::k_del_held<<<num_sms() * 4, 256, 0, s>>>(g->off.p, g->adj.p, udel.p, nud, xflag.p);
    SP_CHECK_LAUNCH();
  }
  if (nua > 0) {
    ingest::k_add_fresh<<<num_sms() * 4, 256, 0, s>>>(g->off.p, g->adj.p, uak.p, nua, udel.p, nud, fresh.p);
    SP_CHECK_LAUNCH();
  }
  {
    size_t t = temp.n;
    SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, t, xflag.p, xrank.p, nud + 1, s));
    t = temp.n;
    SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, t, fresh.p, newrank.p, nua + 1, s));
    g_launches += 2;
  }
  int32_t gone = 0, added = 0;
  SP_TRY(copy_out(&gone, xrank.p + nud, sizeof(int32_t), s));
  SP_TRY(copy_out(&added, newrank.p + nua, sizeof(int32_t), s));
  const int64_t E2 = E - gone + added;
  dbuf<int32_t> off, adj, w;
  SP_TRY(off.alloc((size_t)V + 1));
  SP_TRY(adj.alloc(E2));
  if (g->has_w) SP_TRY(w.alloc(E2));
  if (E > 0) {
    ingest::k_merge_edges<<<num_sms() * 8, 256, 0, s>>>(V, E, g->off.p, g->adj.p, g->has_w ? g->w.p : nullptr,
                                                        udel.p, nud, xrank.p, uak.p, uaw.p, nua, newrank.p, adj.p,
                                                        g->has_w ? w.p : nullptr, cnt.p + 2);
    SP_CHECK_LAUNCH();
  }
  if (added > 0) {
    ingest::k_merge_adds<<<num_sms() * 4, 256, 0, s>>>(g->off.p, g->adj.p, uak.p, uaw.p, nua, newrank.p, udel.p, nud,
                                                       xrank.p, adj.p, g->has_w ? w.p : nullptr);
    SP_CHECK_LAUNCH();
  }
  ingest::k_merge_off<<<num_sms() * 4, 256, 0, s>>>(V, g->off.p, udel.p, nud, xrank.p, uak.p, nua, newrank.p, off.p);
  SP_CHECK_LAUNCH();
  int overflow = 0;
  SP_TRY(copy_out(&overflow, cnt.p + 2, sizeof(int), s));  // synchronises the stream
  if (overflow) {
    set_error("sp_graph_update: an added weight makes an edge's weight leave int32; the graph is unchanged");
    return SP_ERR_INVALID;
  }
  if (held_adds) *held_adds = (int64_t)nua - added;
  // the new CSR replaces the old; plans, the reverse CSR and edgeMap are rebuilt on demand
  free_pr_plan(g->pr);
  free_tc_plan(g->tc);
  free_sssp_plan(g->sssp);
  free_bc_plan(g->bc);
  free_lv_plan(g->lv);
  free_sssp_part_plan(g->sssp_part);
  g->pr = nullptr;
  g->tc = nullptr;
  g->sssp = nullptr;
  g->bc = nullptr;
  g->lv = nullptr;
  g->sssp_part = nullptr;
  g->off.swap(off);
  g->adj.swap(adj);
  if (g->has_w) g->w.swap(w);
  g->roff.release();
  g->radj.release();
  g->emap.release();
  g->has_rev = false;
  g->symmetric = -1;
  g->E = E2;
  return finish_graph(g);
}

}  // namespace sp

extern "C" int sp_graph_update(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                               const int32_t* weight) {
  using namespace sp;
  if (!g || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_graph_update: invalid argument");
    return SP_ERR_INVALID;
  }
  return update_graph(g, n, type, src, dst, weight);
}

extern "C" int sp_graph_export(sp_graph_h g, int32_t* indexofNodes, int32_t* edgeList, int32_t* edgeLen,
                               int32_t* rev_indexofNodes, int32_t* srcList, int32_t* edgeMap) {
  if (!g) {
    set_error("sp_graph_export: NULL graph");
    return SP_ERR_INVALID;
  }
  if (edgeLen && !g->has_w) {
    set_error("sp_graph_export: the graph has no edgeLen");
    return SP_ERR_INVALID;
  }
  if (rev_indexofNodes || srcList) SP_TRY(ensure_reverse(g));
  if (edgeMap) SP_TRY(ensure_emap(g));
  const size_t V1 = (size_t)g->V + 1, E = (size_t)g->E;
  cudaStream_t s = g->stream;
  if (indexofNodes) SP_TRY(copy_out(indexofNodes, g->off.p, 4 * V1, s));
  if (edgeList) SP_TRY(copy_out(edgeList, g->adj.p, 4 * E, s));
  if (edgeLen) SP_TRY(copy_out(edgeLen, g->w.p, 4 * E, s));
  if (rev_indexofNodes) SP_TRY(copy_out(rev_indexofNodes, g->roff.p, 4 * V1, s));
  if (srcList) SP_TRY(copy_out(srcList, g->radj.p, 4 * E, s));
  if (edgeMap) SP_TRY(copy_out(edgeMap, g->emap.p, 4 * E, s));
  return SP_OK;
}
