// Triangle counting for sm_100a.
//
// Semantics: DSL staticDSLCodes/triangle_counting_dsl:1-13 as emitted by the OpenMP
// generator (backend_omp/dsl_cpp_generator.cpp:988-1015, 1277-1299, 2485-2494):
//   count = sum_v sum_{u in N(v), u<v} sum_{w in N(v), w>v} [u->w in E]
// The reference's GPU form tests u->w by binary search (libcuda.cuh:187-212
// findNeighborSorted) from one thread per vertex.
//
// Both paths here are "anchor" loops run by one warp per anchor vertex a:
//   S(a)  = a set staged in a shared-memory hash table (one per warp),
//   P(a)  = probe vertices; for each p in P(a) a probe list L(p) is streamed
//           with all 32 lanes (the (p, element) pairs are flattened across the warp
//           with a prefix sum, so list lengths never idle lanes), and each element
//           is looked up in S(a).
//  * undirected graph (forward CSR == reverse CSR): degree-ordered orientation
//    E+ = {(u,v): (deg u, u) < (deg v, v)}; a = u, S = P = N+(u), L(v) = N+(v).
//    Each triangle is counted once, which equals the formula on a symmetric graph.
//  * any other graph: the formula literally; a = v, S = N(v) ∩ (v, inf),
//    P = N(v) ∩ [0, v), L(u) = N(u) ∩ (v, inf).
// Graphs up to 65536 vertices keep S(a) as a bitmap in shared memory, one per CTA
// of 4 warps that share the anchor's probes (a bitmap per warp held the SM to 24
// resident warps); larger graphs use a per-warp hash table, and anchors whose S does not fit it are counted afterwards
// by whole CTAs with binary search in the sorted global list. Anchors are visited
// heaviest first (estimated probe work) and dealt round-robin to the warps.
//
// Per-vertex counts (PV = true; DSL staticDSLCodes/clustering_coeff:1-14,
// staticClusteringCoeff): every hit of the anchor loop is one triangle (a, p, x),
// found once, and adds one to the counts of all three vertices: x per hit, p by the
// hits of its probe list, a by the hits of all its probe lists. On a symmetric graph
// that is the number of triangles through each vertex, as the DSL's u < v < w loop
// gives; on any other graph the literal-formula path visits exactly the DSL's
// (v, u, w) triples.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "sp_internal.cuh"

namespace sp {

namespace tc {
constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int HCAP = 1024;          // hash slots per warp (load factor <= 1/2)
constexpr int SMAX = HCAP / 2;      // largest S(a) handled by the warp path
constexpr int EMPTY = -1;
constexpr int WU_DEFAULT = 4;       // k_tc_warp: probe-list elements per lane per pass

__device__ __forceinline__ unsigned hslot(int k) { return ((unsigned)k * 2654435761u) >> 22; }  // 10 bits

struct Lists {
  // undirected: o_off/o_adj = oriented CSR; directed: off/adj = forward CSR
  const int32_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  int V;
  int directed;
  int n;  // entries of the anchor order the counting loops visit (V, or a part's share)
};

// S and P ranges of anchor a (as index ranges into adj).
__device__ __forceinline__ void anchor_ranges(const Lists& L, int a, int& sb, int& se, int& pb, int& pe) {
  int b = L.off[a], e = L.off[a + 1];
  if (!L.directed) {
    sb = pb = b;
    se = pe = e;
  } else {
    // first index with adj > a
    int lo = b, hi = e;
    while (lo < hi) {
      int m = (lo + hi) >> 1;
      if (L.adj[m] <= a) lo = m + 1; else hi = m;
    }
    int hi_start = lo;
    // first index with adj >= a
    lo = b;
    hi = hi_start;
    while (lo < hi) {
      int m = (lo + hi) >> 1;
      if (L.adj[m] < a) lo = m + 1; else hi = m;
    }
    pb = b;
    pe = lo;
    sb = hi_start;
    se = e;
  }
}

// Probe list of p for anchor a.
__device__ __forceinline__ void probe_range(const Lists& L, int a, int p, int& lb, int& le) {
  int b = L.off[p], e = L.off[p + 1];
  if (L.directed) {
    int lo = b, hi = e;
    while (lo < hi) {
      int m = (lo + hi) >> 1;
      if (L.adj[m] <= a) lo = m + 1; else hi = m;
    }
    b = lo;
  }
  lb = b;
  le = e;
}

template <bool PV, int WU>
__global__ void __launch_bounds__(THREADS) k_tc_warp(Lists L, const int32_t* __restrict__ order,
                                                     int* __restrict__ heavy, unsigned int* __restrict__ n_heavy,
                                                     unsigned long long* __restrict__ total, int* __restrict__ cf) {
  __shared__ int s_tab[WARPS][HCAP];
  __shared__ short s_slot[WARPS][SMAX];
  __shared__ int s_lb[WARPS][32];
  __shared__ int s_excl[WARPS][32];
  __shared__ int s_p[WARPS][PV ? 32 : 1];
  const int lane = lane_id(), w = warp_id();
  int* tab = s_tab[w];
  for (int i = lane; i < HCAP; i += 32) tab[i] = EMPTY;
  __syncwarp();
  unsigned long long cnt = 0;
  // anchors in decreasing estimated work, dealt round-robin to the warps (no atomics)
  const int gwarp = (blockIdx.x * THREADS + threadIdx.x) >> 5, nwarps = (gridDim.x * THREADS) >> 5;
  for (int ai = gwarp; ai < L.n; ai += nwarps) {
    const int a = order[ai];
    int sb, se, pb, pe;
    anchor_ranges(L, (int)a, sb, se, pb, pe);
    const int ns = se - sb, np = pe - pb;
    if (ns == 0 || np == 0) continue;
    if (ns > SMAX) {
      if (lane == 0) heavy[atomicAdd(n_heavy, 1u)] = (int)a;
      continue;
    }
    // insert S(a)
    for (int i = lane; i < ns; i += 32) {
      int k = L.adj[sb + i];
      unsigned s = hslot(k);
      for (int probe = 0; probe < HCAP; ++probe) {
        int prev = atomicCAS(&tab[s], EMPTY, k);
        if (prev == EMPTY || prev == k) break;
        s = (s + 1) & (HCAP - 1);
      }
      s_slot[w][i] = (short)s;
    }
    __syncwarp();
    unsigned ha = 0;  // PV: this lane's triangles at anchor a
    // probe lists of P(a), 32 probe vertices at a time
    for (int g0 = 0; g0 < np; g0 += 32) {
      int p = g0 + lane < np ? L.adj[pb + g0 + lane] : -1;
      int lb = 0, le = 0;
      if (p >= 0) probe_range(L, (int)a, p, lb, le);
      int len = le - lb;
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      int tot = __shfl_sync(0xffffffffu, incl, 31);
      s_lb[w][lane] = lb;
      s_excl[w][lane] = incl - len;
      if (PV) s_p[w][lane] = p;
      __syncwarp();
      // WU elements per lane per pass: their owners are found and their list entries
      // loaded before any lookup, so the global loads of a pass overlap
      for (int k0 = lane; k0 < tot; k0 += 32 * WU) {
        int xs[WU], own[WU];
#pragma unroll
        for (int q = 0; q < WU; ++q) {
          const int k = k0 + 32 * q;
          xs[q] = -1;
          own[q] = 0;
          if (k < tot) {
            // owner: last lane whose exclusive prefix <= k
            int lo = 0, hi = 31;
            while (lo < hi) {
              int m = (lo + hi + 1) >> 1;
              if (s_excl[w][m] <= k) lo = m; else hi = m - 1;
            }
            own[q] = lo;
            xs[q] = L.adj[s_lb[w][lo] + (k - s_excl[w][lo])];
          }
        }
#pragma unroll
        for (int q = 0; q < WU; ++q) {
          const int x = xs[q];
          if (x < 0) continue;
          unsigned s = hslot(x);
          for (int probe = 0; probe < HCAP; ++probe) {
            int t = tab[s];
            if (t == x) {
              ++cnt;
              if (PV) {
                atomicAdd(cf + x, 1);
                atomicAdd(cf + s_p[w][own[q]], 1);
                ++ha;
              }
              break;
            }
            if (t == EMPTY) break;
            s = (s + 1) & (HCAP - 1);
          }
        }
      }
      __syncwarp();
    }
    if (PV) {
      ha = warp_sum(ha);
      if (lane == 0 && ha) atomicAdd(cf + a, (int)ha);
    }
    // clear the slots S(a) used
    for (int i = lane; i < ns; i += 32) tab[s_slot[w][i]] = EMPTY;
    __syncwarp();
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(total, cnt);
}

// Small graphs (V <= 65536): the same anchor loop with S(a) as a V-bit bitmap per
// warp (8 KB) — a lookup is one shared-memory load and a bit test and any |S(a)|
// fits. Probe lists are long here (about 100 entries on R-MAT 16), so the warp
// streams them one at a time, coalesced, BM_UNROLL loads in flight per lane.
constexpr int BM_WARPS = 4;
constexpr int BM_THREADS = 32 * BM_WARPS;
constexpr int BM_WORDS = 65536 / 32;
constexpr int BM_UNROLL = 4;
constexpr int CTA_WARPS_DEFAULT = 4;  // k_tc_bitmap_cta warps per CTA: 0.173 ms on R-MAT 16 vs 0.209 per-warp
// Per-vertex counts in k_tc_bitmap_cta: anchors with at most CNT_SLOTS elements in S(a)
// count hits per element in shared memory (16-bit halves of 32-bit words; a count is at
// most |P(a)| < 65536 since P(a) holds distinct vertex ids below 65536) and add them to
// cf once per (anchor, element) afterwards.
constexpr int CNT_SLOTS = 4096;

__global__ void __launch_bounds__(BM_THREADS) k_tc_bitmap(Lists L, const int32_t* __restrict__ order,
                                                          unsigned long long* __restrict__ total) {
  __shared__ unsigned s_bm[BM_WARPS][BM_WORDS];
  const int lane = lane_id(), w = warp_id();
  unsigned* bm = s_bm[w];
  for (int i = lane; i < BM_WORDS; i += 32) bm[i] = 0u;
  __syncwarp();
  unsigned long long cnt = 0;
  const int gwarp = (blockIdx.x * BM_THREADS + threadIdx.x) >> 5, nwarps = (gridDim.x * BM_THREADS) >> 5;
  for (int ai = gwarp; ai < L.n; ai += nwarps) {
    const int a = order[ai];
    int sb, se, pb, pe;
    anchor_ranges(L, a, sb, se, pb, pe);
    const int ns = se - sb, np = pe - pb;
    if (ns == 0 || np == 0) continue;
    for (int i = lane; i < ns; i += 32) {
      const int k = L.adj[sb + i];
      atomicOr(&bm[k >> 5], 1u << (k & 31));
    }
    __syncwarp();
    // probe lists: bounds of 32 probe vertices per lane load, then the whole warp
    // streams one list at a time (coalesced, BM_UNROLL loads in flight per lane)
    for (int g0 = 0; g0 < np; g0 += 32) {
      const int p = g0 + lane < np ? L.adj[pb + g0 + lane] : -1;
      int lb = 0, le = 0;
      if (p >= 0) probe_range(L, a, p, lb, le);
      const int nl = min(32, np - g0);
      for (int l = 0; l < nl; ++l) {
        const int b = __shfl_sync(0xffffffffu, lb, l);
        const int e = __shfl_sync(0xffffffffu, le, l);
        for (int k0 = b + lane; k0 < e; k0 += 32 * BM_UNROLL) {
          int x[BM_UNROLL];
#pragma unroll
          for (int u = 0; u < BM_UNROLL; ++u) {
            const int k = k0 + 32 * u;
            x[u] = k < e ? __ldg(L.adj + k) : -1;
          }
#pragma unroll
          for (int u = 0; u < BM_UNROLL; ++u)
            if (x[u] >= 0) cnt += (bm[x[u] >> 5] >> (x[u] & 31)) & 1u;
        }
      }
    }
    __syncwarp();
    for (int i = lane; i < ns; i += 32) bm[L.adj[sb + i] >> 5] = 0u;
    __syncwarp();
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(total, cnt);
}

// CTA-wide form of k_tc_bitmap: one bitmap per CTA of NW warps, so shared memory no
// longer caps the resident warps (8 KB per CTA instead of per warp). The CTA takes
// one anchor at a time (LPT order, dealt round-robin to CTAs); warp w takes the
// probes w, w + NW, ... of it, 32 probe ranges per lane load, and streams each
// list across its lanes. The bitmap is set, probed and cleared between barriers.
template <int NW, int MINB, bool PV>
__global__ void __launch_bounds__(NW * 32, MINB) k_tc_bitmap_cta(Lists L, const int32_t* __restrict__ order,
                                                                 unsigned long long* __restrict__ total,
                                                                 int* __restrict__ cf) {
  __shared__ unsigned s_bm[BM_WORDS];
  __shared__ unsigned short s_pre[PV ? BM_WORDS : 1];    // PV: set bits in the words before each word
  __shared__ unsigned s_cnt[PV ? CNT_SLOTS / 2 : 1];      // PV: hits per element of S(a), two per word
  __shared__ unsigned s_wsum[PV ? NW : 1];
  constexpr int NT = NW * 32;
  constexpr int WPT = BM_WORDS / NT;  // bitmap words per thread in the prefix count
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < BM_WORDS; i += NT) s_bm[i] = 0u;
  if (PV)
    for (int i = tid; i < CNT_SLOTS / 2; i += NT) s_cnt[i] = 0u;
  __syncthreads();
  unsigned long long cnt = 0;
  for (int ai = blockIdx.x; ai < L.n; ai += gridDim.x) {
    const int a = order[ai];
    int sb, se, pb, pe;
    anchor_ranges(L, a, sb, se, pb, pe);
    const int ns = se - sb, np = pe - pb;
    if (ns == 0 || np == 0) continue;  // the same for every thread of the CTA
    for (int i = tid; i < ns; i += NT) {
      const int k = L.adj[sb + i];
      atomicOr(&s_bm[k >> 5], 1u << (k & 31));
    }
    __syncthreads();
    // PV: element x of S(a) is slot s_pre[x / 32] + (set bits of its word below x) of
    // the sorted S(a); its hits are counted in shared memory when S(a) fits
    const bool priv = PV && ns <= CNT_SLOTS;  // the same for every thread of the CTA
    if (priv) {
      unsigned c = 0;
#pragma unroll
      for (int j = 0; j < WPT; ++j) c += __popc(s_bm[tid * WPT + j]);
      unsigned incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_wsum[w] = incl;
      __syncthreads();
      unsigned base = incl - c;
      for (int k = 0; k < w; ++k) base += s_wsum[k];
#pragma unroll
      for (int j = 0; j < WPT; ++j) {
        s_pre[tid * WPT + j] = (unsigned short)base;
        base += __popc(s_bm[tid * WPT + j]);
      }
      __syncthreads();
    }
    unsigned ha = 0;  // PV: this warp's triangles at anchor a (lane 0)
    for (int g0 = 0; w + NW * g0 < np; g0 += 32) {
      const int pi = w + NW * (g0 + lane);
      const int p = pi < np ? L.adj[pb + pi] : -1;
      int lb = 0, le = 0;
      if (p >= 0) probe_range(L, a, p, lb, le);
      const int nl = min(32, (np - w + NW - 1) / NW - g0);
      for (int l = 0; l < nl; ++l) {
        const int b = __shfl_sync(0xffffffffu, lb, l);
        const int e = __shfl_sync(0xffffffffu, le, l);
        unsigned hp = 0;  // PV: this lane's hits in the probe list of lane l's vertex
        for (int k0 = b + lane; k0 < e; k0 += 32 * BM_UNROLL) {
          int x[BM_UNROLL];
#pragma unroll
          for (int u = 0; u < BM_UNROLL; ++u) {
            const int k = k0 + 32 * u;
            x[u] = k < e ? __ldg(L.adj + k) : -1;
          }
#pragma unroll
          for (int u = 0; u < BM_UNROLL; ++u)
            if (x[u] >= 0) {
              const unsigned hit = (s_bm[x[u] >> 5] >> (x[u] & 31)) & 1u;
              cnt += hit;
              if (PV && hit) {
                if (priv) {
                  const int xw = x[u] >> 5;
                  const unsigned slot = s_pre[xw] + __popc(s_bm[xw] & ((1u << (x[u] & 31)) - 1u));
                  atomicAdd(&s_cnt[slot >> 1], 1u << ((slot & 1u) * 16u));
                } else {
                  atomicAdd(cf + x[u], 1);
                }
                ++hp;
              }
            }
        }
        if (PV) {
          const int pl = __shfl_sync(0xffffffffu, p, l);
          hp = warp_sum(hp);
          if (lane == 0 && hp) atomicAdd(cf + pl, (int)hp);
          ha += hp;
        }
      }
    }
    if (PV && lane == 0 && ha) atomicAdd(cf + a, (int)ha);
    __syncthreads();
    if (priv) {
      for (int i = tid; i < ns; i += NT) {
        const unsigned c = (s_cnt[i >> 1] >> ((i & 1) * 16)) & 0xffffu;
        if (c) atomicAdd(cf + L.adj[sb + i], (int)c);
      }
      __syncthreads();
      for (int i = tid; i < (ns + 1) / 2; i += NT) s_cnt[i] = 0u;
    }
    for (int i = tid; i < ns; i += NT) s_bm[L.adj[sb + i] >> 5] = 0u;
    __syncthreads();
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(total, cnt);
}

// Heavy anchors: one CTA each, lookups by binary search in the sorted S(a).
template <bool PV>
__global__ void __launch_bounds__(THREADS) k_tc_heavy(Lists L, const int* __restrict__ heavy,
                                                      const unsigned int* __restrict__ n_heavy,
                                                      unsigned long long* __restrict__ total, int* __restrict__ cf) {
  __shared__ int s_lb[THREADS];
  __shared__ int s_excl[THREADS];
  __shared__ int s_p[PV ? THREADS : 1];
  __shared__ int s_tot;
  __shared__ unsigned long long s_red[WARPS];
  const int nh = (int)*n_heavy;
  unsigned long long cnt = 0;
  for (int h = blockIdx.x; h < nh; h += gridDim.x) {
    const int a = heavy[h];
    int sb, se, pb, pe;
    anchor_ranges(L, a, sb, se, pb, pe);
    unsigned long long ha = 0;  // PV: this thread's triangles at anchor a
    for (int g0 = pb; g0 < pe; g0 += THREADS) {
      int p = g0 + (int)threadIdx.x < pe ? L.adj[g0 + threadIdx.x] : -1;
      int lb = 0, le = 0;
      if (p >= 0) probe_range(L, a, p, lb, le);
      int len = le - lb;
      // block exclusive scan of len
      typedef cub::BlockScan<int, THREADS> Scan;
      __shared__ typename Scan::TempStorage ts;
      int excl, tot;
      Scan(ts).ExclusiveSum(len, excl, tot);
      s_lb[threadIdx.x] = lb;
      s_excl[threadIdx.x] = excl;
      if (PV) s_p[threadIdx.x] = p;
      if (threadIdx.x == 0) s_tot = tot;
      __syncthreads();
      for (int k = threadIdx.x; k < s_tot; k += THREADS) {
        int lo = 0, hi = THREADS - 1;
        while (lo < hi) {
          int m = (lo + hi + 1) >> 1;
          if (s_excl[m] <= k) lo = m; else hi = m - 1;
        }
        int x = L.adj[s_lb[lo] + (k - s_excl[lo])];
        int l = sb, r = se;
        while (l < r) {
          int m = (l + r) >> 1;
          if (L.adj[m] < x) l = m + 1; else r = m;
        }
        if (l < se && L.adj[l] == x) {
          ++cnt;
          if (PV) {
            atomicAdd(cf + x, 1);
            atomicAdd(cf + s_p[lo], 1);
            ++ha;
          }
        }
      }
      __syncthreads();
    }
    if (PV) {
      ha = block_sum<THREADS>(ha, s_red);
      if (threadIdx.x == 0 && ha) atomicAdd(cf + a, (int)ha);
    }
  }
  cnt = block_sum<THREADS>(cnt, s_red);
  if (threadIdx.x == 0 && cnt) atomicAdd(total, cnt);
}

// Plain form: the generated CUDA code's shape — one thread per vertex v, the
// formula's double loop over N(v), u->w tested by binary search in N(u)
// (libcuda.cuh:187-212 findNeighborSorted).
__global__ void k_tc_plain(const int32_t* __restrict__ off, const int32_t* __restrict__ adj, int V,
                           unsigned long long* __restrict__ total) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  unsigned long long c = 0;
  for (int e = off[v]; e < off[v + 1]; ++e) {
    int u = adj[e];
    if (u >= v) continue;
    for (int e2 = off[v]; e2 < off[v + 1]; ++e2) {
      int w = adj[e2];
      if (w <= v) continue;
      int lo = off[u], hi = off[u + 1] - 1;
      while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int x = adj[mid];
        if (x == w) {
          ++c;
          break;
        }
        if (x < w) lo = mid + 1; else hi = mid - 1;
      }
    }
  }
  if (c) atomicAdd(total, c);
}

// Plain per-vertex form: the generated CUDA shape of staticClusteringCoeff (one
// thread per vertex v, the double loop over N(v), u->w by binary search in N(u)),
// each triangle adding one to cf of v, u and w.
__global__ void k_lcc_plain(const int32_t* __restrict__ off, const int32_t* __restrict__ adj, int V,
                            int* __restrict__ cf) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  for (int e = off[v]; e < off[v + 1]; ++e) {
    int u = adj[e];
    if (u >= v) continue;
    for (int e2 = off[v]; e2 < off[v + 1]; ++e2) {
      int w = adj[e2];
      if (w <= v) continue;
      int lo = off[u], hi = off[u + 1] - 1;
      while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int x = adj[mid];
        if (x == w) {
          atomicAdd(cf + v, 1);
          atomicAdd(cf + u, 1);
          atomicAdd(cf + w, 1);
          break;
        }
        if (x < w) lo = mid + 1; else hi = mid - 1;
      }
    }
  }
}

// Estimated work of anchor a: the probe-list lengths it streams (sum over P(a)),
// as a sort key (negated, so an ascending sort puts the heaviest first).
__global__ void k_tc_work(Lists L, int32_t* __restrict__ key, int32_t* __restrict__ id) {
  const int lane = threadIdx.x & 31;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < L.V; a += (gridDim.x * blockDim.x) >> 5) {
    int sb, se, pb, pe;
    anchor_ranges(L, a, sb, se, pb, pe);
    long long w = 0;
    for (int i = pb + lane; i < pe; i += 32) {
      const int p = L.adj[i];
      w += L.off[p + 1] - L.off[p];
    }
    w = warp_sum(w);
    if (lane == 0) {
      key[a] = (int32_t)(-min(w * (long long)(se - sb > 0), (long long)INT32_MAX));
      id[a] = a;
    }
  }
}

// Orientation: keep v in N+(u) iff (deg u, u) < (deg v, v).
__device__ __forceinline__ bool before(int du, int u, int dv, int v) { return du < dv || (du == dv && u < v); }

// Edge-parallel orientation (tiles of EDGE_TILE entries): keep[i] = 1 when edge i
// (u -> v) is kept in N+(u). A scan of keep gives each kept edge its place in the
// oriented CSR in row order, and ooff[u] is the scan at u's first edge. One warp per
// vertex took 3.6 ms on undirected R-MAT 20, most of it the hub rows' tails.
__global__ void k_orient_flag(int V, long long E, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                              int32_t* __restrict__ keep) {
  __shared__ int s_v[2];
  for (long long t0 = (long long)blockIdx.x * EDGE_TILE; t0 < E; t0 += (long long)gridDim.x * EDGE_TILE) {
    const long long t1 = t0 + EDGE_TILE < E ? t0 + EDGE_TILE : E;
    if (threadIdx.x < 2) s_v[threadIdx.x] = edge_source(off, 0, V, threadIdx.x == 0 ? t0 : t1 - 1);
    __syncthreads();
    const int vlo = s_v[0], vhi = s_v[1];
    for (long long i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
      const int u = edge_source(off, vlo, vhi + 1, i);
      const int v = adj[i];
      keep[i] = before(off[u + 1] - off[u], u, off[v + 1] - off[v], v) ? 1 : 0;
    }
    __syncthreads();
  }
}

__global__ void k_orient_off(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ pos,
                             int32_t* __restrict__ ooff) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u <= V; u += gridDim.x * blockDim.x) ooff[u] = pos[off[u]];
}

__global__ void k_orient_scatter(long long E, const int32_t* __restrict__ adj, const int32_t* __restrict__ pos,
                                 int32_t* __restrict__ oadj) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (long long)gridDim.x * blockDim.x)
    if (pos[i + 1] > pos[i]) oadj[pos[i]] = adj[i];
}

// Part `part` of `nparts`: every nparts-th anchor of the heaviest-first order, starting at
// position part (n = ceil((V - part) / nparts) entries, so part + (n - 1) * nparts < V).
__global__ void k_order_part(const int32_t* __restrict__ order, int n, int part, int nparts,
                             int32_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = order[part + i * nparts];
}

// ---- batches of edge updates on a symmetric graph (DynTC's Batch block)
__device__ __forceinline__ unsigned long long ukey(int a, int b) {
  const unsigned lo = (unsigned)min(a, b), hi = (unsigned)max(a, b);
  return ((unsigned long long)lo << 32) | hi;
}

__device__ __forceinline__ bool in_sorted(const unsigned long long* __restrict__ s, int n, unsigned long long k) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (s[m] < k) lo = m + 1; else hi = m;
  }
  return lo < n && s[lo] == k;
}

// x in the sorted row adj[b .. e)
__device__ __forceinline__ bool in_row(const int32_t* __restrict__ adj, int b, int e, int x) {
  int lo = b, hi = e;
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (adj[m] < x) lo = m + 1; else hi = m;
  }
  return lo < e && adj[lo] == x;
}

// Triangles of a symmetric CSR through the undirected edges keys[0 .. n) (lo << 32 | hi,
// lo < hi, sorted, distinct), in two kernels. k_tri_work gives each edge (a, b) its work,
// the length of the shorter of the two rows (0 when check is set and (a, b) is not an
// edge; its two other edges, found in both rows, always are). After a scan of the work,
// k_tri_flat gives every (edge, entry of its shorter row) pair one thread, which
// searches the longer row for that third vertex c: an edge between two hubs is spread
// over as many threads as its shorter row has entries. A triangle holding k of the edges
// is found once from each of them, so cnt[k - 1] counts finds and the triangles number
// cnt[0] + cnt[1] / 2 + cnt[2] / 3.
__global__ void k_tri_work(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                           const unsigned long long* __restrict__ keys, int n, int check,
                           unsigned long long* __restrict__ work) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    const int a = (int)(k >> 32), b = (int)(k & 0xffffffffull);
    const int ab = off[a], ae = off[a + 1], bb = off[b], be = off[b + 1];
    work[i] = check && !in_row(adj, ab, ae, b) ? 0ull : (unsigned long long)min(ae - ab, be - bb);
  }
}

// delta (optional): each triangle adds `sign` to its three vertices once, from the find
// whose edge (a, b) has the smallest key among the triangle's edges in keys.
__global__ void k_tri_flat(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                           const unsigned long long* __restrict__ keys, int n,
                           const unsigned long long* __restrict__ pre, unsigned long long total,
                           unsigned long long* __restrict__ cnt, int* __restrict__ delta, int sign) {
  unsigned long long c1 = 0, c2 = 0, c3 = 0;
  const unsigned long long step = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += step) {
    // the edge i with pre[i] <= t < pre[i + 1] (pre[0] = 0, pre[n] = total)
    int lo = 0, hi = n;
    while (hi - lo > 1) {
      const int m = (lo + hi) >> 1;
      if (pre[m] <= t) lo = m; else hi = m;
    }
    const unsigned long long k = keys[lo];
    const int a = (int)(k >> 32), b = (int)(k & 0xffffffffull);
    const int ab = off[a], ae = off[a + 1], bb = off[b], be = off[b + 1];
    const bool a_short = ae - ab <= be - bb;
    const int c = adj[(a_short ? ab : bb) + (int)(t - pre[lo])];
    if (c == a || c == b || !in_row(adj, a_short ? bb : ab, a_short ? be : ae, c)) continue;
    const unsigned long long kac = ukey(a, c), kbc = ukey(b, c);
    const bool sac = in_sorted(keys, n, kac), sbc = in_sorted(keys, n, kbc);
    const int m = 1 + (int)sac + (int)sbc;
    c1 += m == 1;
    c2 += m == 2;
    c3 += m == 3;
    if (delta && (!sac || k < kac) && (!sbc || k < kbc)) {
      atomicAdd(&delta[a], sign);
      atomicAdd(&delta[b], sign);
      atomicAdd(&delta[c], sign);
    }
  }
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  c3 = warp_sum(c3);
  if ((threadIdx.x & 31) == 0 && (c1 | c2 | c3)) {
    atomicAdd(&cnt[0], c1);
    atomicAdd(&cnt[1], c2);
    atomicAdd(&cnt[2], c3);
  }
}

__global__ void k_add_i32(int n, const int* __restrict__ d, int32_t* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += d[i];
}

// Additions that add an edge: absent from the CSR before the batch, or deleted by it.
__global__ void k_new_edges(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const unsigned long long* __restrict__ add, int na,
                            const unsigned long long* __restrict__ del, int nd, unsigned char* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
    const unsigned long long k = add[i];
    const int a = (int)(k >> 32), b = (int)(k & 0xffffffffull);
    flag[i] = !in_row(adj, off[a], off[a + 1], b) || in_sorted(del, nd, k);
  }
}

}  // namespace tc

struct TcPlan {
  dbuf<int32_t> ooff, oadj;  // oriented CSR (undirected graphs)
  dbuf<int32_t> order;       // anchors, heaviest first
  dbuf<int> heavy;
  dbuf<unsigned int> ctr;    // [0] next anchor, [1] heavy count
  dbuf<unsigned long long> total;
  bool oriented = false;
  bool built = false;
  // learned variant inputs (vstat < 0: not yet) and the learned choice under model var_gen
  int vstat = -1;
  int64_t vmax = 0, vsq = 0, vheavy = 0;
  int var_choice = -1;
  unsigned var_gen = 0;
};

int tc_cta_warps_default() { return tc::CTA_WARPS_DEFAULT; }

void free_tc_plan(TcPlan* p) {
  if (!p) return;
  p->ooff.release();
  p->oadj.release();
  p->order.release();
  p->heavy.release();
  p->ctr.release();
  p->total.release();
  delete p;
}

static int build_tc_plan(sp_graph* g) {
  if (g->tc && g->tc->built) return SP_OK;
  if (g->tc) {
    free_tc_plan(g->tc);
    g->tc = nullptr;
  }
  SP_TRY(ensure_symmetry(g));
  TcPlan* p = new TcPlan();
  cudaStream_t s = g->stream;
  auto fail = [&](int st) {
    free_tc_plan(p);
    return st;
  };
  int st;
  if ((st = p->heavy.alloc(g->V)) || (st = p->ctr.alloc(2)) || (st = p->total.alloc(1))) return fail(st);
  if (g->symmetric == 1) {
    if ((st = p->ooff.alloc(g->V + 1))) return fail(st);
    const long long E = g->E;
    dbuf<int32_t> keep, pos;
    if ((st = keep.alloc(E + 1)) || (st = pos.alloc(E + 1))) return fail(st);
    cudaMemsetAsync(keep.p + E, 0, sizeof(int32_t), s);
    if (E > 0) {
      tc::k_orient_flag<<<num_sms() * 8, 256, 0, s>>>(g->V, E, g->off.p, g->adj.p, keep.p);
      g_launches++;
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, keep.p, pos.p, (int)(E + 1), s);
    dbuf<unsigned char> tmp;
    if ((st = tmp.alloc(tb))) return fail(st);
    cub::DeviceScan::ExclusiveSum(tmp.p, tb, keep.p, pos.p, (int)(E + 1), s);
    g_launches++;
    tc::k_orient_off<<<num_sms() * 4, 256, 0, s>>>(g->V, g->off.p, pos.p, p->ooff.p);
    g_launches++;
    int32_t eplus = 0;
    if ((st = copy_out(&eplus, p->ooff.p + g->V, sizeof(int32_t), s))) return fail(st);
    if ((st = p->oadj.alloc(eplus))) return fail(st);
    if (E > 0) {
      tc::k_orient_scatter<<<num_sms() * 8, 256, 0, s>>>(E, g->adj.p, pos.p, p->oadj.p);
      g_launches++;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("tc orientation: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(SP_ERR_CUDA);
    }
    p->oriented = true;
  }
  {
    tc::Lists L;
    L.V = g->V;
    L.directed = p->oriented ? 0 : 1;
    L.off = p->oriented ? p->ooff.p : g->off.p;
    L.adj = p->oriented ? p->oadj.p : g->adj.p;
    L.n = g->V;
    dbuf<int32_t> key, id, skey;
    if ((st = key.alloc(g->V)) || (st = id.alloc(g->V)) || (st = skey.alloc(g->V)) || (st = p->order.alloc(g->V)))
      return fail(st);
    tc::k_tc_work<<<num_sms() * 8, 256, 0, s>>>(L, key.p, id.p);
    g_launches++;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, skey.p, id.p, p->order.p, g->V, 0, 32, s);
    dbuf<unsigned char> tmp;
    if ((st = tmp.alloc(tb))) return fail(st);
    cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, skey.p, id.p, p->order.p, g->V, 0, 32, s);
    g_launches++;
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("tc anchor order: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(SP_ERR_CUDA);
    }
  }
  p->built = true;
  g->tc = p;
  return SP_OK;
}

static tc::Lists tc_lists(sp_graph* g, int n) {
  TcPlan* p = g->tc;
  tc::Lists L;
  L.V = g->V;
  L.directed = p->oriented ? 0 : 1;
  L.off = p->oriented ? p->ooff.p : g->off.p;
  L.adj = p->oriented ? p->oadj.p : g->adj.p;
  L.n = n;
  return L;
}

// ---- learned kernel variant -------------------------------------------------------
// Graphs up to 65536 vertices choose the shared-bitmap kernel's CTA width (0 = a bitmap
// per warp); larger graphs choose the hash kernel's probe-list elements per lane per
// pass. Entries 2 and 7 are the fixed defaults.
namespace tc {
struct Variant {
  int bitmap, cta_warps, wu;
};
constexpr Variant VARIANTS[] = {{1, 0, 0}, {1, 2, 0}, {1, 4, 0}, {1, 8, 0},
                                {1, 16, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 4}};
constexpr int N_VARIANTS = (int)(sizeof(VARIANTS) / sizeof(VARIANTS[0]));
constexpr int DEFAULT_BITMAP = 2, DEFAULT_HASH = 7;
}  // namespace tc

int tc_variant_count() { return tc::N_VARIANTS; }

// Inputs: graph shape, symmetry, the path (bitmap below 65537 vertices), the share of
// entries in rows above the hash path's set size, then the candidate.
int tc_variant_features(sp_graph* g, int cand, float* x, int* applicable) {
  if (cand < 0 || cand >= tc::N_VARIANTS) return SP_ERR_INVALID;
  SP_TRY(build_tc_plan(g));
  TcPlan* p = g->tc;
  if (p->vstat < 0) {
    const int thr[1] = {tc::SMAX};
    DegStats ds;
    SP_TRY(degree_stats(g->off.p, g->V, thr, 1, g->stream, &ds));
    p->vmax = ds.max_deg;
    p->vsq = ds.sum_sq;
    p->vheavy = ds.edges_above[0];
    p->vstat = 1;
  }
  const tc::Variant& c = tc::VARIANTS[cand];
  const bool bitmap_path = g->V <= 65536;
  const double V = g->V, E = std::max<double>(1.0, (double)g->E), avg = E / std::max(1.0, V);
  const double lcw = std::log2(1.0 + c.cta_warps);
  x[0] = (float)std::log2(std::max(1.0, V));
  x[1] = (float)std::log2(E + 1.0);
  x[2] = (float)avg;
  x[3] = (float)std::log2((double)p->vmax + 1.0);
  x[4] = (float)std::log2((double)p->vsq / E + 1.0);
  x[5] = (float)(g->symmetric > 0);
  x[6] = bitmap_path ? 1.0f : 0.0f;
  x[7] = (float)((double)p->vheavy / E);
  x[8] = (float)c.bitmap;
  x[9] = (float)lcw;
  x[10] = (c.bitmap && c.cta_warps == 0) ? 1.0f : 0.0f;
  x[11] = c.wu ? (float)std::log2((double)c.wu) : 0.0f;
  x[12] = (float)(lcw * avg / 16.0);
  *applicable = (c.bitmap != 0) == bitmap_path;
  return SP_OK;
}

static int tc_variant_pick(sp_graph* g, int* cand) {
  *cand = -1;
  const int mode = g->variant[VAR_TC];
  if (mode >= 0) {
    if ((tc::VARIANTS[mode].bitmap != 0) != (g->V <= 65536)) {
      set_error("tc.variant %d does not apply to a graph of %d vertices", mode, g->V);
      return SP_ERR_INVALID;
    }
    *cand = mode;
    return SP_OK;
  }
  if (mode != -1 || g->tc_cta_warps >= 0 || g->tc_unroll > 0) return SP_OK;
  const unsigned gen = variant_generation(VAR_TC);
  if (!gen) return SP_OK;
  TcPlan* p = g->tc;
  if (p->var_gen == gen && p->var_choice >= 0) {
    *cand = p->var_choice;
    return SP_OK;
  }
  std::vector<float> X((size_t)tc::N_VARIANTS * SP_MLP_IN);
  std::vector<int> ok(tc::N_VARIANTS);
  for (int k = 0; k < tc::N_VARIANTS; ++k) SP_TRY(tc_variant_features(g, k, X.data() + (size_t)k * SP_MLP_IN, &ok[k]));
  int best = -1;
  const int st = variant_choose(VAR_TC, X, ok, g->V <= 65536 ? tc::DEFAULT_BITMAP : tc::DEFAULT_HASH, g->stream, &best);
  if (st == SP_ERR_UNSUPPORTED) return SP_OK;
  SP_TRY(st);
  p->var_choice = best;
  p->var_gen = gen;
  *cand = best;
  return SP_OK;
}

// Triangles anchored at order[0 .. n) (the whole count when order is the plan's and n = V).
static int tc_count(sp_graph* g, const int32_t* order, int n, int64_t* triangle_count) {
  TcPlan* p = g->tc;
  cudaStream_t s = g->stream;
  const tc::Lists L = tc_lists(g, n);
  SP_CHECK_CUDA(cudaMemsetAsync(p->ctr.p, 0, sizeof(unsigned int) * 2, s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->total.p, 0, sizeof(unsigned long long), s));
  int cta_warps = g->tc_cta_warps >= 0 ? g->tc_cta_warps : tc::CTA_WARPS_DEFAULT;
  int wu = g->tc_unroll > 0 ? g->tc_unroll : tc::WU_DEFAULT;
  int cand = -1;
  SP_TRY(tc_variant_pick(g, &cand));
  if (cand >= 0) {
    if (tc::VARIANTS[cand].bitmap) cta_warps = tc::VARIANTS[cand].cta_warps;
    else wu = tc::VARIANTS[cand].wu;
  }
  g->last_variant[VAR_TC] = cand;
  if (g->V <= 65536 && cta_warps > 0) {
    void (*k)(tc::Lists, const int32_t*, unsigned long long*, int*) =
        cta_warps == 2   ? tc::k_tc_bitmap_cta<2, 24, false>
        : cta_warps == 4 ? tc::k_tc_bitmap_cta<4, 16, false>
        : cta_warps == 8 ? tc::k_tc_bitmap_cta<8, 8, false>
                         : tc::k_tc_bitmap_cta<16, 4, false>;
    int per_sm = 0;
    SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, cta_warps * 32, 0));
    k<<<num_sms() * std::max(1, per_sm), cta_warps * 32, 0, s>>>(L, order, p->total.p, nullptr);
    SP_CHECK_LAUNCH();
  } else if (g->V <= 65536) {
    int per_sm = 0;
    SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc::k_tc_bitmap, tc::BM_THREADS, 0));
    tc::k_tc_bitmap<<<num_sms() * std::max(1, per_sm), tc::BM_THREADS, 0, s>>>(L, order, p->total.p);
    SP_CHECK_LAUNCH();
  } else {
    void (*k)(tc::Lists, const int32_t*, int*, unsigned int*, unsigned long long*, int*) =
        wu == 1 ? tc::k_tc_warp<false, 1> : wu == 2 ? tc::k_tc_warp<false, 2> : tc::k_tc_warp<false, 4>;
    k<<<num_sms() * 4, tc::THREADS, 0, s>>>(L, order, p->heavy.p, p->ctr.p + 1, p->total.p, nullptr);
    SP_CHECK_LAUNCH();
    tc::k_tc_heavy<false><<<num_sms() * 2, tc::THREADS, 0, s>>>(L, p->heavy.p, p->ctr.p + 1, p->total.p, nullptr);
    SP_CHECK_LAUNCH();
  }
  unsigned long long h = 0;
  SP_TRY(copy_out(&h, p->total.p, sizeof(h), s));
  *triangle_count = (int64_t)h;
  return SP_OK;
}

// Per-vertex triangle counts of the triangles anchored at order[0 .. n), added to counts.
static int lcc_count(sp_graph* g, const int32_t* order, int n, int* counts) {
  TcPlan* p = g->tc;
  cudaStream_t s = g->stream;
  const tc::Lists L = tc_lists(g, n);
  SP_CHECK_CUDA(cudaMemsetAsync(p->ctr.p, 0, sizeof(unsigned int) * 2, s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->total.p, 0, sizeof(unsigned long long), s));
  if (g->V <= 65536) {
    int per_sm = 0;
    SP_CHECK_CUDA(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc::k_tc_bitmap_cta<4, 8, true>, 4 * 32, 0));
    tc::k_tc_bitmap_cta<4, 8, true><<<num_sms() * std::max(1, per_sm), 4 * 32, 0, s>>>(L, order, p->total.p, counts);
    SP_CHECK_LAUNCH();
  } else {
    tc::k_tc_warp<true, tc::WU_DEFAULT>
        <<<num_sms() * 4, tc::THREADS, 0, s>>>(L, order, p->heavy.p, p->ctr.p + 1, p->total.p, counts);
    SP_CHECK_LAUNCH();
    tc::k_tc_heavy<true><<<num_sms() * 2, tc::THREADS, 0, s>>>(L, p->heavy.p, p->ctr.p + 1, p->total.p, counts);
    SP_CHECK_LAUNCH();
  }
  return SP_OK;
}

// The anchors of part `part` of `nparts` (every nparts-th of the heaviest-first order) in
// out, their number in n. The plan must be built.
static int order_part(sp_graph* g, int part, int nparts, dbuf<int32_t>& out, int& n) {
  n = part < g->V ? (g->V - part + nparts - 1) / nparts : 0;
  SP_TRY(out.alloc(std::max(1, n)));
  if (n > 0) {
    tc::k_order_part<<<num_sms() * 4, 256, 0, g->stream>>>(g->tc->order.p, n, part, nparts, out.p);
    SP_CHECK_LAUNCH();
  }
  return SP_OK;
}

}  // namespace sp

extern "C" int sp_tc(sp_graph_h g, int64_t* triangle_count, int32_t variant) {
  using namespace sp;
  if (!g || !triangle_count) {
    set_error("sp_tc: NULL argument");
    return SP_ERR_INVALID;
  }
  if (variant == SP_TC_PLAIN) {
    if (!g->tc) g->tc = new TcPlan();
    TcPlan* p = g->tc;
    SP_TRY(p->total.alloc(1));
    SP_CHECK_CUDA(cudaMemsetAsync(p->total.p, 0, sizeof(unsigned long long), g->stream));
    const int tb = 512;  // backend_cuda/dsl_cpp_generator.cpp:56-77
    tc::k_tc_plain<<<(g->V + tb - 1) / tb, tb, 0, g->stream>>>(g->off.p, g->adj.p, g->V, p->total.p);
    SP_CHECK_LAUNCH();
    unsigned long long h = 0;
    SP_TRY(copy_out(&h, p->total.p, sizeof(h), g->stream));
    *triangle_count = (int64_t)h;
    return SP_OK;
  }
  if (variant != SP_TC_TUNED) {
    set_error("sp_tc: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  SP_TRY(build_tc_plan(g));
  return tc_count(g, g->tc->order.p, g->V, triangle_count);
}

extern "C" int sp_clustering_coeff(sp_graph_h g, int32_t* cf, int32_t variant) {
  using namespace sp;
  if (!g || !cf) {
    set_error("sp_clustering_coeff: NULL argument");
    return SP_ERR_INVALID;
  }
  if (variant != SP_TC_TUNED && variant != SP_TC_PLAIN) {
    set_error("sp_clustering_coeff: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  dbuf<int> counts;
  SP_TRY(counts.alloc(g->V));
  if (g->V) SP_CHECK_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * g->V, s));
  if (variant == SP_TC_PLAIN) {
    const int tb = 512;  // backend_cuda/dsl_cpp_generator.cpp:56-77
    if (g->V) {
      tc::k_lcc_plain<<<(g->V + tb - 1) / tb, tb, 0, s>>>(g->off.p, g->adj.p, g->V, counts.p);
      SP_CHECK_LAUNCH();
    }
    return copy_out(cf, counts.p, sizeof(int32_t) * g->V, s);
  }
  SP_TRY(build_tc_plan(g));
  SP_TRY(lcc_count(g, g->tc->order.p, g->V, counts.p));
  return copy_out(cf, counts.p, sizeof(int32_t) * g->V, s);
}

// Anchor parts for several GPUs: part r of n counts the triangles anchored at every n-th
// vertex of the heaviest-first anchor order, starting at position r, so the parts' work
// is dealt like the single-GPU kernels deal it to warps and every triangle falls in
// exactly one part. The parts' counts add up to sp_tc's, and their per-vertex vectors
// to sp_clustering_coeff's. The reference's multi-GPU generator gives each device the
// contiguous vertex range [i V / n, (i + 1) V / n) of every forall instead
// (backend_multigpu/dsl_cpp_generator.cpp:4286-4288), which on R-MAT puts the hubs, and
// most of the work, in the first range.
static int check_part(const char* fn, sp_graph_h g, const void* out, int32_t part, int32_t nparts) {
  if (!g || !out) {
    sp::set_error("%s: NULL argument", fn);
    return SP_ERR_INVALID;
  }
  if (nparts < 1 || part < 0 || part >= nparts) {
    sp::set_error("%s: part %d of %d", fn, part, nparts);
    return SP_ERR_INVALID;
  }
  return SP_OK;
}

extern "C" int sp_tc_part(sp_graph_h g, int32_t part, int32_t nparts, int64_t* triangle_count) {
  using namespace sp;
  SP_TRY(check_part("sp_tc_part", g, triangle_count, part, nparts));
  SP_TRY(build_tc_plan(g));
  if (nparts == 1) return tc_count(g, g->tc->order.p, g->V, triangle_count);
  dbuf<int32_t> mine;
  int n = 0;
  SP_TRY(order_part(g, part, nparts, mine, n));
  return tc_count(g, mine.p, n, triangle_count);
}

extern "C" int sp_clustering_coeff_part(sp_graph_h g, int32_t part, int32_t nparts, int32_t* cf) {
  using namespace sp;
  SP_TRY(check_part("sp_clustering_coeff_part", g, cf, part, nparts));
  cudaStream_t s = g->stream;
  dbuf<int> counts;
  SP_TRY(counts.alloc(g->V));
  if (g->V) SP_CHECK_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * g->V, s));
  SP_TRY(build_tc_plan(g));
  dbuf<int32_t> mine;
  int n = g->V;
  const int32_t* order = g->tc->order.p;
  if (nparts > 1) {
    SP_TRY(order_part(g, part, nparts, mine, n));
    order = mine.p;
  }
  SP_TRY(lcc_count(g, order, n, counts.p));
  return copy_out(cf, counts.p, sizeof(int32_t) * g->V, s);
}

namespace sp {

// Triangles of g's CSR through the sorted undirected keys d_keys[0 .. n).
// delta (optional, int32[V] on the device): each triangle adds sign to its vertices.
static int tri_through(sp_graph* g, const unsigned long long* d_keys, int n, int check, int64_t* out,
                       int* delta = nullptr, int sign = 0) {
  *out = 0;
  if (n == 0) return SP_OK;
  cudaStream_t s = g->stream;
  dbuf<unsigned long long> cnt, work, pre;
  dbuf<unsigned char> temp;
  SP_TRY(cnt.alloc(3));
  SP_TRY(work.alloc((size_t)n + 1));
  SP_TRY(pre.alloc((size_t)n + 1));
  SP_CHECK_CUDA(cudaMemsetAsync(cnt.p, 0, 3 * sizeof(unsigned long long), s));
  SP_CHECK_CUDA(cudaMemsetAsync(work.p + n, 0, sizeof(unsigned long long), s));
  tc::k_tri_work<<<std::min(num_sms() * 4, (n + 255) / 256), 256, 0, s>>>(g->off.p, g->adj.p, d_keys, n, check,
                                                                          work.p);
  SP_CHECK_LAUNCH();
  size_t tb = 0;
  SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, work.p, pre.p, n + 1, s));
  SP_TRY(temp.alloc(std::max<size_t>(1, tb)));
  SP_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, work.p, pre.p, n + 1, s));
  g_launches++;
  unsigned long long total = 0;
  SP_TRY(copy_out(&total, pre.p + n, sizeof(total), s));
  if (total > 0) {
    const unsigned long long want = (total + 255) / 256;
    const int blocks = (int)std::min<unsigned long long>(want, (unsigned long long)num_sms() * 16);
    tc::k_tri_flat<<<blocks, 256, 0, s>>>(g->off.p, g->adj.p, d_keys, n, pre.p, total, cnt.p, delta, sign);
    SP_CHECK_LAUNCH();
  }
  unsigned long long h[3];
  SP_TRY(copy_out(h, cnt.p, sizeof(h), s));
  if (h[1] % 2 || h[2] % 3) {
    set_error("sp_tc_dynamic: %llu / %llu finds of triangles with two / three batch edges", h[1], h[2]);
    return SP_ERR_UNSUPPORTED;
  }
  *out = (int64_t)(h[0] + h[1] / 2 + h[2] / 3);
  return SP_OK;
}

// Sorted distinct directed keys of one update type, and whether that set is symmetric.
static bool symmetric_set(std::vector<unsigned long long>& k) {
  std::sort(k.begin(), k.end());
  k.erase(std::unique(k.begin(), k.end()), k.end());
  std::vector<unsigned long long> t(k.size());
  for (size_t i = 0; i < k.size(); ++i) t[i] = (k[i] << 32) | (k[i] >> 32);
  std::sort(t.begin(), t.end());
  return t == k;
}

// One batch on g (deletions, then additions) with the triangles it changes. On a
// symmetric graph whose batch keeps it symmetric (incremental = true):
//   T(new) = T(old) - [triangles of the old graph through deleted edges]
//                   + [triangles of the new graph through added edges],
// where a deleted edge is one the old graph holds and an added edge one the graph
// lacks after the deletions; dcount gets the difference and delta (optional, int32[V]
// on the device, zeroed) the per-vertex differences. Otherwise the batch is only
// applied (incremental = false). A bad update is reported with g unchanged.
static int batch_triangles(sp_graph* g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                           const int32_t* weight, int64_t* dcount, int* delta, bool& incremental) {
  *dcount = 0;
  incremental = false;
  std::vector<unsigned long long> dd, ad, du, au;  // directed keys; undirected keys (lo < hi)
  for (int64_t i = 0; i < n; ++i) {
    const int32_t a = src[i], b = dst[i];
    if ((type[i] != 'a' && type[i] != 'd') || a < 0 || a >= g->V || b < 0 || b >= g->V)
      return update_graph(g, n, type, src, dst, weight);  // reports the bad update, changes nothing
    const unsigned long long k = ((unsigned long long)(uint32_t)a << 32) | (uint32_t)b;
    const unsigned long long u = ((unsigned long long)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
    (type[i] == 'd' ? dd : ad).push_back(k);
    if (a != b) (type[i] == 'd' ? du : au).push_back(u);
  }
  SP_TRY(ensure_symmetry(g));
  if (!(g->symmetric == 1 && symmetric_set(dd) && symmetric_set(ad))) return update_graph(g, n, type, src, dst, weight);
  for (auto* v : {&du, &au}) {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
  }
  const int nd = (int)du.size(), na = (int)au.size();
  cudaStream_t s = g->stream;
  dbuf<unsigned long long> d_del, d_add, d_new;
  dbuf<unsigned char> flag, temp;
  dbuf<int> d_nnew;
  SP_TRY(d_del.alloc(std::max(1, nd)));
  SP_TRY(d_add.alloc(std::max(1, na)));
  SP_TRY(d_new.alloc(std::max(1, na)));
  SP_TRY(flag.alloc(std::max(1, na)));
  SP_TRY(d_nnew.alloc(1));
  if (nd) SP_CHECK_CUDA(cudaMemcpyAsync(d_del.p, du.data(), 8 * (size_t)nd, cudaMemcpyHostToDevice, s));
  if (na) SP_CHECK_CUDA(cudaMemcpyAsync(d_add.p, au.data(), 8 * (size_t)na, cudaMemcpyHostToDevice, s));
  int64_t lost = 0, gained = 0;
  SP_TRY(tri_through(g, d_del.p, nd, 1, &lost, delta, -1));
  int nnew = 0;
  if (na) {
    tc::k_new_edges<<<num_sms() * 4, 256, 0, s>>>(g->off.p, g->adj.p, d_add.p, na, d_del.p, nd, flag.p);
    SP_CHECK_LAUNCH();
    size_t tb = 0;
    SP_CHECK_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, d_add.p, flag.p, d_new.p, d_nnew.p, na, s));
    SP_TRY(temp.alloc(std::max<size_t>(1, tb)));
    SP_CHECK_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, d_add.p, flag.p, d_new.p, d_nnew.p, na, s));
    g_launches++;
    SP_TRY(copy_out(&nnew, d_nnew.p, sizeof(int), s));
  }
  SP_TRY(update_graph(g, n, type, src, dst, weight));
  g->symmetric = 1;  // a symmetric graph minus and plus symmetric edge sets
  SP_TRY(tri_through(g, d_new.p, nnew, 0, &gained, delta, 1));
  *dcount = gained - lost;
  incremental = true;
  return SP_OK;
}

}  // namespace sp

// DynTC's Batch block (dynamicDSLCodes/dynamicBatchTCV2:142-199): the batch is applied
// (deletions, then additions) and the count updated. On a symmetric graph with a batch
// that keeps it symmetric, only triangles through changed edges are counted; a
// triangle through k changed edges is found k times and weighted 1/k, as the DSL's
// count1/2 + count2/4 + count3/6 does for updates given in both directions. Otherwise
// the updated graph is counted again.
extern "C" int sp_tc_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                             const int32_t* weight, int64_t* triangle_count) {
  using namespace sp;
  if (!g || !triangle_count || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_tc_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  g->tc_last_incremental = 1;
  if (n == 0) return SP_OK;  // nothing changed: the caller's count stands
  int64_t dcount = 0;
  bool incremental = false;
  SP_TRY(batch_triangles(g, n, type, src, dst, weight, &dcount, nullptr, incremental));
  g->tc_last_incremental = incremental ? 1 : 0;
  if (incremental) {
    *triangle_count += dcount;
    return SP_OK;
  }
  SP_TRY(build_tc_plan(g));
  return tc_count(g, g->tc->order.p, g->V, triangle_count);
}

// DynCF's Batch block (dynamicDSLCodes/dynamicBatchClustering:44-53): the batch, then
// cf[V] (host or device; staticClusteringCoeff's counts before the batch on entry)
// brought up to date. Incremental on a symmetric graph with a symmetric batch, as for
// sp_tc_dynamic, each changed triangle adding -1 or +1 to its three vertices once;
// otherwise the updated graph is counted again.
extern "C" int sp_clustering_coeff_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src,
                                           const int32_t* dst, const int32_t* weight, int32_t* cf) {
  using namespace sp;
  if (!g || !cf || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_clustering_coeff_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  g->tc_last_incremental = 1;
  if (n == 0) return SP_OK;
  cudaStream_t s = g->stream;
  dbuf<int> delta;
  SP_TRY(delta.alloc(std::max(1, g->V)));
  if (g->V) SP_CHECK_CUDA(cudaMemsetAsync(delta.p, 0, sizeof(int) * g->V, s));
  int64_t dcount = 0;
  bool incremental = false;
  SP_TRY(batch_triangles(g, n, type, src, dst, weight, &dcount, delta.p, incremental));
  g->tc_last_incremental = incremental ? 1 : 0;
  if (incremental) {
    dbuf<int32_t> x;
    SP_TRY(x.alloc(std::max(1, g->V)));
    SP_CHECK_CUDA(cudaMemcpyAsync(x.p, cf, sizeof(int32_t) * g->V, cudaMemcpyDefault, s));
    tc::k_add_i32<<<num_sms() * 4, 256, 0, s>>>(g->V, delta.p, x.p);
    SP_CHECK_LAUNCH();
    return copy_out(cf, x.p, sizeof(int32_t) * g->V, s);
  }
  SP_CHECK_CUDA(cudaMemsetAsync(delta.p, 0, sizeof(int) * g->V, s));
  SP_TRY(build_tc_plan(g));
  SP_TRY(lcc_count(g, g->tc->order.p, g->V, delta.p));
  return copy_out(cf, delta.p, sizeof(int32_t) * g->V, s);
}
