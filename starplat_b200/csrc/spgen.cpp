// Seeded synthetic graph generators and CSR construction (host, C++17 + OpenMP).
//
// The reference builds its CSR container from a text edge list in
// graphcode/graph.hpp:464-859 (duplicates merged with summed weights, adjacency
// sorted by destination, reverse CSR with sorted sources). That parser is
// O(indeg^2) per vertex and cannot reach the benchmark sizes (R-MAT scale 22/23),
// so graphs are generated here directly as edge lists and turned into exactly the
// same CSR layout: forward CSR sorted by destination, reverse CSR sorted by source,
// int32 indices, duplicates removed.
//
// Every random draw is a pure function of (seed, edge index), so the same graph is
// produced regardless of thread count, on any machine.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// Uniform integer in [0, n) from 32 random bits (multiply-shift).
inline uint32_t bounded32(uint32_t r, uint32_t n) {
  return (uint32_t)(((uint64_t)r * (uint64_t)n) >> 32);
}

inline double unit_double(uint64_t r) {  // [0,1)
  return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

template <class T>
inline T fetch_add(T* p, T v) {
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}

// Exclusive prefix sum of counts[0..n) into off[0..n]; returns the total.
int64_t exclusive_scan(const int32_t* counts, int64_t n, int64_t* off) {
  int64_t s = 0;
  for (int64_t i = 0; i < n; ++i) {
    off[i] = s;
    s += counts[i];
  }
  off[n] = s;
  return s;
}

}  // namespace

extern "C" {

// R-MAT edge list: nedges pairs over 2^scale vertices with quadrant
// probabilities (a, b, c, 1-a-b-c). Vertex ids are used as generated (no
// permutation). Returns nedges.
int64_t spg_rmat_edges(int scale, int64_t nedges, double a, double b, double c,
                       uint64_t seed, int32_t* src, int32_t* dst) {
  const uint64_t ta = (uint64_t)(a * 4294967296.0);
  const uint64_t tb = (uint64_t)((a + b) * 4294967296.0);
  const uint64_t tc = (uint64_t)((a + b + c) * 4294967296.0);
  const uint64_t base = splitmix64(seed ^ 0x5250414D47454E31ULL);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nedges; ++i) {
    uint64_t st = splitmix64(base + (uint64_t)i * 0xD1B54A32D192ED03ULL);
    uint32_t s = 0, d = 0;
    uint64_t word = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) {
        st = splitmix64(st);
        word = st;
      }
      uint64_t r = (l & 1) ? (word >> 32) : (word & 0xFFFFFFFFULL);
      uint32_t sb, db;
      if (r < ta) {
        sb = 0; db = 0;
      } else if (r < tb) {
        sb = 0; db = 1;
      } else if (r < tc) {
        sb = 1; db = 0;
      } else {
        sb = 1; db = 1;
      }
      s |= sb << (scale - 1 - l);
      d |= db << (scale - 1 - l);
    }
    src[i] = (int32_t)s;
    dst[i] = (int32_t)d;
  }
  return nedges;
}

// Erdos-Renyi G(n, m): m uniform random ordered pairs over [0, n).
int64_t spg_er_edges(int32_t n, int64_t m, uint64_t seed, int32_t* src, int32_t* dst) {
  const uint64_t base = splitmix64(seed ^ 0x45524E4D47454E32ULL);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    uint64_t r = splitmix64(base + (uint64_t)i * 0xD1B54A32D192ED03ULL);
    src[i] = (int32_t)bounded32((uint32_t)r, (uint32_t)n);
    dst[i] = (int32_t)bounded32((uint32_t)(r >> 32), (uint32_t)n);
  }
  return m;
}

// Block boundaries of a planted partition with power-law block sizes:
// raw sizes x_k = (1-U)^(-1/(exponent-1)) (density ~ x^-exponent, x >= 1),
// scaled to sum to V with every block at least min_size vertices.
// Writes block_start[0..nblocks]; returns 0 on success.
int32_t spg_sbm_blocks(int32_t V, int32_t nblocks, double exponent, int32_t min_size,
                       uint64_t seed, int32_t* block_start) {
  if (nblocks <= 0 || (int64_t)nblocks * min_size > V || exponent <= 1.0) return -1;
  std::vector<double> x(nblocks);
  double tot = 0;
  uint64_t st = splitmix64(seed ^ 0x53424D424C4B5333ULL);
  for (int k = 0; k < nblocks; ++k) {
    st = splitmix64(st);
    double u = unit_double(st);
    x[k] = std::pow(1.0 - u, -1.0 / (exponent - 1.0));
    tot += x[k];
  }
  const int64_t spare = (int64_t)V - (int64_t)nblocks * min_size;
  std::vector<int64_t> sz(nblocks);
  int64_t used = 0;
  int kmax = 0;
  for (int k = 0; k < nblocks; ++k) {
    sz[k] = min_size + (int64_t)std::floor(x[k] / tot * (double)spare);
    used += sz[k];
    if (x[k] > x[kmax]) kmax = k;
  }
  sz[kmax] += (int64_t)V - used;  // rounding remainder goes to the largest block
  block_start[0] = 0;
  for (int k = 0; k < nblocks; ++k) block_start[k + 1] = block_start[k] + (int32_t)sz[k];
  return 0;
}

// Planted-partition edges: for pair i, u is uniform over [0, V); with
// probability p_in v is uniform inside u's block, otherwise uniform over the
// vertices outside it. Every vertex therefore has the same expected degree.
int64_t spg_sbm_edges(int32_t V, int32_t nblocks, const int32_t* block_start, int64_t m,
                      double p_in, uint64_t seed, int32_t* src, int32_t* dst) {
  const uint64_t base = splitmix64(seed ^ 0x53424D4544474534ULL);
  const uint64_t tin = (uint64_t)(p_in * 4294967296.0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    uint64_t r0 = splitmix64(base + (uint64_t)i * 0xD1B54A32D192ED03ULL);
    uint64_t r1 = splitmix64(r0);
    uint32_t u = bounded32((uint32_t)r0, (uint32_t)V);
    int32_t blk = (int32_t)(std::upper_bound(block_start, block_start + nblocks + 1, (int32_t)u) -
                            block_start) - 1;
    int32_t bs = block_start[blk], bz = block_start[blk + 1] - block_start[blk];
    uint32_t v;
    if ((r0 >> 32) < tin || bz == V) {
      v = (uint32_t)bs + bounded32((uint32_t)r1, (uint32_t)bz);
    } else {
      v = bounded32((uint32_t)r1, (uint32_t)(V - bz));
      if ((int32_t)v >= bs) v += (uint32_t)bz;
    }
    src[i] = (int32_t)u;
    dst[i] = (int32_t)v;
  }
  return m;
}

// Forward CSR from an edge list: optional symmetrisation (both directions) and
// self-loop removal; duplicates are removed and each adjacency is sorted by
// destination (graph.hpp:725-733). off has V+1 entries; adj has room for cap
// entries (M, or 2M when symmetrising). Returns E, or -1 if E would not fit
// int32 offsets or cap is too small.
int64_t spg_csr_from_edges(int32_t V, int64_t M, const int32_t* src, const int32_t* dst,
                           int symmetrize, int drop_self, int32_t* off, int32_t* adj,
                           int64_t cap) {
  const int64_t need = symmetrize ? 2 * M : M;
  if (cap < need) return -1;
  std::vector<int32_t> cnt(V, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    int32_t s = src[i], d = dst[i];
    if (drop_self && s == d) continue;
    fetch_add(&cnt[s], 1);
    if (symmetrize) fetch_add(&cnt[d], 1);
  }
  std::vector<int64_t> pos(V + 1);
  exclusive_scan(cnt.data(), V, pos.data());
  std::vector<int64_t> cur(pos.begin(), pos.end() - 1);
  // Scatter into adj (used as scratch), then sort + unique each segment.
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    int32_t s = src[i], d = dst[i];
    if (drop_self && s == d) continue;
    int64_t p = fetch_add(&cur[s], (int64_t)1);
    adj[p] = d;
    if (symmetrize) {
      int64_t q = fetch_add(&cur[d], (int64_t)1);
      adj[q] = s;
    }
  }
  std::vector<int32_t> uniq(V, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < V; ++v) {
    int32_t* b = adj + pos[v];
    int32_t* e = adj + pos[v + 1];
    std::sort(b, e);
    uniq[v] = (int32_t)(std::unique(b, e) - b);
  }
  std::vector<int64_t> npos(V + 1);
  int64_t E = exclusive_scan(uniq.data(), V, npos.data());
  if (E >= (int64_t)INT32_MAX) return -1;
  // Compact in place: segments only move left, process in order.
  for (int32_t v = 0; v < V; ++v) {
    if (npos[v] != pos[v]) std::memmove(adj + npos[v], adj + pos[v], sizeof(int32_t) * uniq[v]);
  }
  for (int32_t v = 0; v <= V; ++v) off[v] = (int32_t)npos[v];
  return E;
}

// Reverse CSR (graph.hpp:781-833): roff[V+1], radj[E] = sources of the in-edges
// of each vertex, sorted ascending. Optional emap[E] gives, for each reverse
// entry, the index of the same edge in the forward CSR (graph.hpp:836-846).
void spg_transpose(int32_t V, int64_t E, const int32_t* off, const int32_t* adj,
                   int32_t* roff, int32_t* radj, int32_t* emap) {
  std::vector<int32_t> cnt(V, 0);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < E; ++e) fetch_add(&cnt[adj[e]], 1);
  std::vector<int64_t> pos(V + 1);
  exclusive_scan(cnt.data(), V, pos.data());
  for (int32_t v = 0; v <= V; ++v) roff[v] = (int32_t)pos[v];
  // Sequential-in-source scatter per thread chunk keeps work simple; the
  // per-vertex sort afterwards makes the result independent of thread timing.
  std::vector<int64_t> cur(pos.begin(), pos.end() - 1);
  std::vector<int64_t> tmp_e;
  if (emap) tmp_e.resize(E);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t u = 0; u < V; ++u) {
    for (int32_t e = off[u]; e < off[u + 1]; ++e) {
      int32_t v = adj[e];
      int64_t p = fetch_add(&cur[v], (int64_t)1);
      radj[p] = u;
      if (emap) tmp_e[p] = e;
    }
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < V; ++v) {
    int64_t b = pos[v], e = pos[v + 1];
    if (!emap) {
      std::sort(radj + b, radj + e);
    } else {
      std::vector<std::pair<int32_t, int64_t>> seg;
      seg.reserve(e - b);
      for (int64_t i = b; i < e; ++i) seg.emplace_back(radj[i], tmp_e[i]);
      std::sort(seg.begin(), seg.end());
      for (int64_t i = b; i < e; ++i) {
        radj[i] = seg[i - b].first;
        emap[i] = (int32_t)seg[i - b].second;
      }
    }
  }
}

// Integer edge weights in [wmin, wmax], a hash of (seed, u, v). With
// symmetric != 0 the hash uses (min(u,v), max(u,v)) so both directions of an
// undirected edge carry the same weight.
void spg_weights_hash(int32_t V, int64_t E, const int32_t* off, const int32_t* adj,
                      uint64_t seed, int32_t wmin, int32_t wmax, int symmetric, int32_t* w) {
  const uint64_t span = (uint64_t)((int64_t)wmax - (int64_t)wmin + 1);
  const uint64_t base = splitmix64(seed ^ 0x5745494748545335ULL);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t u = 0; u < V; ++u) {
    for (int32_t e = off[u]; e < off[u + 1]; ++e) {
      uint32_t a = (uint32_t)u, b = (uint32_t)adj[e];
      if (symmetric && a > b) std::swap(a, b);
      uint64_t h = splitmix64(base ^ (((uint64_t)a << 32) | b));
      w[e] = (int32_t)((int64_t)wmin + (int64_t)(((h >> 32) * span) >> 32));
    }
  }
}

// rows x cols 4-neighbour grid, both directions, vertex id = r*cols + c.
// Adjacency is sorted: up, left, right, down. Returns E.
int64_t spg_grid(int32_t rows, int32_t cols, int32_t* off, int32_t* adj) {
  const int64_t V = (int64_t)rows * cols;
  std::vector<int32_t> deg(V);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < V; ++v) {
    int32_t r = (int32_t)(v / cols), c = (int32_t)(v % cols);
    deg[v] = (r > 0) + (c > 0) + (c + 1 < cols) + (r + 1 < rows);
  }
  int64_t s = 0;
  for (int64_t v = 0; v < V; ++v) {
    off[v] = (int32_t)s;
    s += deg[v];
  }
  off[V] = (int32_t)s;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < V; ++v) {
    int32_t r = (int32_t)(v / cols), c = (int32_t)(v % cols);
    int64_t p = off[v];
    if (r > 0) adj[p++] = (int32_t)(v - cols);
    if (c > 0) adj[p++] = (int32_t)(v - 1);
    if (c + 1 < cols) adj[p++] = (int32_t)(v + 1);
    if (r + 1 < rows) adj[p++] = (int32_t)(v + cols);
  }
  return s;
}

// Writes a CSR as a text edge list, one "src dst weight" line per edge in CSR order
// (the format graph::parseGraph reads). Lines are formatted in parallel blocks and
// written in order. Returns the bytes written, or -1 if the file cannot be written.
int64_t spg_write_edgelist(const char* path, int32_t V, const int32_t* off, const int32_t* adj, const int32_t* w) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  const int64_t E = off[V];
  const int64_t B = 1 << 20;  // edges per block
  const int64_t nb = (E + B - 1) / B;
  int64_t total = 0;
  std::vector<std::string> out(16);
  for (int64_t b0 = 0; b0 < nb; b0 += 16) {
    const int64_t b1 = std::min(nb, b0 + 16);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = b0; b < b1; ++b) {
      std::string& s = out[b - b0];
      s.clear();
      const int64_t e0 = b * B, e1 = std::min(E, e0 + B);
      // the source of e0: last v with off[v] <= e0
      int64_t lo = 0, hi = V;
      while (lo < hi) {
        const int64_t m = (lo + hi + 1) / 2;
        if (off[m] <= e0) lo = m; else hi = m - 1;
      }
      int32_t u = (int32_t)lo;
      char tmp[48];
      for (int64_t e = e0; e < e1; ++e) {
        while (off[u + 1] <= e) ++u;
        const int n = snprintf(tmp, sizeof(tmp), "%d %d %d\n", u, adj[e], w ? w[e] : 1);
        s.append(tmp, n);
      }
    }
    for (int64_t b = b0; b < b1; ++b) {
      const std::string& s = out[b - b0];
      if (fwrite(s.data(), 1, s.size(), f) != s.size()) {
        fclose(f);
        return -1;
      }
      total += (int64_t)s.size();
    }
  }
  fclose(f);
  return total;
}

// Is the forward CSR equal to its reverse (an undirected graph)?
int32_t spg_is_symmetric(int32_t V, const int32_t* off, const int32_t* adj,
                         const int32_t* roff, const int32_t* radj) {
  int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (int32_t v = 0; v <= V; ++v)
    if (off[v] != roff[v]) bad |= 1;
  if (bad) return 0;
  const int64_t E = off[V];
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (int64_t e = 0; e < E; ++e)
    if (adj[e] != radj[e]) bad |= 1;
  return bad ? 0 : 1;
}

int32_t spg_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
