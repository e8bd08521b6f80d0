// Louvain community detection (local move + aggregation) for sm_100a.
//
// Semantics: DSL staticDSLCodes/community_detection:1-211 (the reference's only
// Louvain DSL; MPI-only there) and the runnable CUDA restatement
// dynamic_louvain_community_detection/communitydetection_sequential_allocation.cu
// (computeGraphWeight :746-778, modularity :1060-1080):
//   W = sum of all directed edge weights; k_v = weighted degree (+ self-loop weight);
//   gain(v -> c) = k_{v,c} - tot_c * k_v / W   (tot_c without v for v's own community,
//   community_detection:83-107); Q = sum_c in_c / W - (tot_c / W)^2 (:40);
//   local moves repeat while Q improves by more than `threshold`, then communities
//   become vertices (self-loop = internal weight) and the whole repeats while a level
//   improves Q by more than `threshold` (:34, :111, :208).
// The sequential order of the DSL cannot be kept on a GPU, so results are compared
// on modularity (within 1e-3 of the sequential restatement), not on labels.
//
// B200 design:
//  * synchronous local moves: every vertex of a sub-sweep picks its best community
//    from the same snapshot; two sub-sweeps per sweep (vertex hash parity) and the
//    singleton rule (a singleton moves to another singleton only if that label is
//    smaller) keep neighbours from swapping back and forth;
//  * per-vertex neighbour-community weights by degree bin: up to 64 edges, one warp
//    with no table (lanes holding one community found by __match_any_sync and summed
//    by shuffles); up to slots / 2, one CTA with a hash table of up to `slots` entries
//    in dynamic shared memory (16384 by default; per level, the learned variant may
//    take 1024, 2048 or 4096, which fit more CTAs per SM); above that, one CTA with a
//    table in global scratch; FP64 values, shared-memory atomics in the tables;
//  * vertices binned by degree class and by sub-sweep parity, so a sub-sweep's
//    kernels read only the vertices that may move in it;
//  * tot_c with FP64 atomics aggregated per warp over lanes of one community (exact
//    for integer weights); Q from the total internal weight (a CTA reduction) and
//    the tot_c;
//  * aggregation: communities renumbered densely, external edges emitted at scan
//    positions with the key c_u * C + c_v, sorted by this library's stable LSD radix
//    sort (sp_prims.cuh), and each run of equal keys summed by one warp in a fixed
//    order (so the next level's weights do not depend on scheduling).

#include <climits>
#include <cstring>
#include <cmath>
#include <vector>

#include "sp_internal.cuh"
#include "sp_mlp_dev.cuh"
#include "sp_prims.cuh"

namespace sp {

namespace lv {
constexpr int THREADS = 256;
constexpr int WARP_DEG = 64;
constexpr int CTA_SLOTS_MAX = 16384;
constexpr int EMPTY = -1;

__device__ __forceinline__ unsigned hmix(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

struct Level {
  int n;
  const int32_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  const double* __restrict__ w;
  const double* __restrict__ sl;  // self-loop weight per vertex
  int unit;                       // 1: every w is 1.0 (the input graph without weights), not read
};

struct MoveArgs {
  Level L;
  const int32_t* __restrict__ comm;
  const double* __restrict__ tot;
  const int32_t* __restrict__ csize;
  const double* __restrict__ kv;
  int32_t* newcomm;
  const int32_t* __restrict__ list;  // vertices of this bin
  int nlist;
  int parity;     // sub-sweep: vertices with hmix(v)&1 == parity
  double W;
  double* gtab_val;  // global tables (big bin)
  int32_t* gtab_key;
  const int64_t* gtab_off;  // per list entry: table offset (big bin)
};

// insert (key, val) into an open-addressing table; returns false if full
__device__ __forceinline__ bool tab_add(int32_t* keys, double* vals, unsigned mask, int key, double val) {
  unsigned s = hmix((unsigned)key) & mask;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    int prev = atomicCAS(&keys[s], EMPTY, key);
    if (prev == EMPTY || prev == key) {
      atomicAdd(&vals[s], val);
      return true;
    }
    s = (s + 1) & mask;
  }
  return false;
}

// better candidate: larger gain; on a tie the current community, then the smaller id
__device__ __forceinline__ bool better(double g1, int c1, double g2, int c2, int cur) {
  if (g1 != g2) return g1 > g2;
  if (c1 == cur) return true;
  if (c2 == cur) return false;
  return c1 < c2;
}

// tot_cv, size_cv: tot[cv] and csize[cv], which a caller can load early.
__device__ __forceinline__ int decide(const MoveArgs& a, int cv, double kv, double tot_cv, int size_cv,
                                      double best_gain, int best_c) {
  // baseline: the DSL starts from currcommunity.kin (always 0) - tot' * k_v / W (:88)
  const double stay = 0.0 - (tot_cv - kv) * kv / a.W;
  if (best_c < 0 || !(best_gain > stay) || best_c == cv) return cv;
  if (size_cv == 1 && a.csize[best_c] == 1 && best_c > cv) return cv;  // singleton rule
  return best_c;
}

// Weight of the community c, summed over the lanes of grp (the lanes holding c) in
// lane order; every lane of grp gets the sum.
__device__ __forceinline__ double group_sum(unsigned grp, double w) {
  double s = 0.0;
  for (unsigned m = grp; m; m &= m - 1) s += __shfl_sync(grp, w, __ffs(m) - 1);
  return s;
}

// A weight w for which 32 * w and every partial sum of up to 32 copies are exact in FP64
// (an integer of magnitude below 2^40), so a group of k lanes sums to k * w in any order.
__device__ __forceinline__ bool uniform_ok(double w) { return w == rint(w) && fabs(w) < 1099511627776.0; }

// One warp per vertex of degree <= 64 (= WARP_DEG), no tables: a lane holds one
// neighbour per 32-edge round; __match_any_sync groups the lanes holding the same
// community and the group sums its weights in lane order; a round-1 group adds into
// the round-0 group of the same community, or stands as a candidate of its own. Every
// distinct neighbour community is scored once, with the tables' gain and tie-break.
// The warp's next list entry, and tot / csize of v's own community, are loaded ahead of
// their use, so they add no round trip to the chain of dependent loads of a vertex
// (SBM 1M: 28.1 -> 27.7 ms for the whole Louvain, A/B on one box; 45 registers, and
// held to 40 it measured the same as before).
__global__ void __launch_bounds__(THREADS) k_move_warp(MoveArgs a) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * THREADS + threadIdx.x) >> 5, nw = (gridDim.x * THREADS) >> 5;
  int vnext = gw < a.nlist ? a.list[gw] : 0;
  for (int i = gw; i < a.nlist; i += nw) {
    const int v = vnext;
    if (i + nw < a.nlist) vnext = a.list[i + nw];
    const int cv = a.comm[v];
    const double kv = a.kv[v];
    const int b = a.L.off[v], e = a.L.off[v + 1];
    const double tot_cv = a.tot[cv];
    const int size_cv = a.csize[cv];
    const int j0 = b + lane, j1 = b + 32 + lane;
    const bool on0 = j0 < e, on1 = j1 < e;
    const int c0 = on0 ? a.comm[a.L.adj[j0]] : -1 - lane;  // idle lanes: keys no community has
    const double w0 = on0 ? (a.L.unit ? 1.0 : a.L.w[j0]) : 0.0;
    const unsigned g0 = __match_any_sync(0xffffffffu, c0);
    // When every edge of the round carries the same integer weight (unit weights, the
    // usual case), a group's lane-order sum is its size times that weight, exactly: the
    // product gives the same value without a shuffle per group member.
    const double wr0 = __shfl_sync(0xffffffffu, w0, 0);
    const bool uni0 = a.L.unit || (__all_sync(0xffffffffu, !on0 || w0 == wr0) && uniform_ok(wr0));
    double s0 = uni0 ? (double)__popc(g0) * wr0 : group_sum(g0, w0);
    const bool lead0 = on0 && lane == __ffs(g0) - 1;
    bool cand1 = false;
    int c1 = -1;
    double s1 = 0.0;
    if (e - b > 32) {  // the same for the whole warp
      c1 = on1 ? a.comm[a.L.adj[j1]] : -33 - lane;
      const double w1 = on1 ? (a.L.unit ? 1.0 : a.L.w[j1]) : 0.0;
      const unsigned g1 = __match_any_sync(0xffffffffu, c1);
      const double wr1 = __shfl_sync(0xffffffffu, w1, 0);
      const bool uni1 = a.L.unit || (__all_sync(0xffffffffu, !on1 || w1 == wr1) && uniform_ok(wr1));
      s1 = uni1 ? (double)__popc(g1) * wr1 : group_sum(g1, w1);
      cand1 = on1 && lane == __ffs(g1) - 1;
      unsigned leads = __ballot_sync(0xffffffffu, cand1);
      while (leads) {
        const int l = __ffs(leads) - 1;
        leads &= leads - 1;
        const int cl = __shfl_sync(0xffffffffu, c1, l);
        const double sl = __shfl_sync(0xffffffffu, s1, l);
        const bool hit = lead0 && c0 == cl;
        if (hit) s0 += sl;
        if (__any_sync(0xffffffffu, hit) && lane == l) cand1 = false;
      }
    }
    double bg = -INFINITY;
    int bc = -1;
    if (lead0) {
      const double tc = (c0 == cv) ? tot_cv - kv : a.tot[c0];
      bg = s0 - tc * kv / a.W;
      bc = c0;
    }
    if (cand1) {
      const double tc = (c1 == cv) ? tot_cv - kv : a.tot[c1];
      const double gain = s1 - tc * kv / a.W;
      if (bc < 0 || better(gain, c1, bg, bc, cv)) {
        bg = gain;
        bc = c1;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double og = __shfl_xor_sync(0xffffffffu, bg, o);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
      if (oc >= 0 && (bc < 0 || better(og, oc, bg, bc, cv))) {
        bg = og;
        bc = oc;
      }
    }
    if (lane == 0) a.newcomm[v] = decide(a, cv, kv, tot_cv, size_cv, bg, bc);
  }
}

// Plain form (SP_LV_PLAIN): one thread per vertex of the sub-sweep's parity and no
// tables. Each neighbour community is scored once, at the first neighbour carrying it,
// and its weight k_{v,c} is found by rescanning the neighbour list: O(deg^2) work per
// vertex, the shape of the reference's runnable CUDA local move
// (communitydetection_sequential_allocation.cu, moveNodesKernel). Gains, tie-breaks and
// the singleton rule are the tuned kernels' own, so with integer weights both forms
// make the same moves.
__global__ void k_move_plain(MoveArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.L.n || (int)(hmix((unsigned)v) & 1u) != a.parity) return;
  const int cv = a.comm[v];
  const double kv = a.kv[v];
  const int b = a.L.off[v], e = a.L.off[v + 1];
  double bg = -INFINITY;
  int bc = -1;
  for (int j = b; j < e; ++j) {
    const int c = a.comm[a.L.adj[j]];
    bool seen = false;
    for (int i = b; i < j && !seen; ++i) seen = a.comm[a.L.adj[i]] == c;
    if (seen) continue;
    double kc = 0.0;
    for (int i = b; i < e; ++i)
      if (a.comm[a.L.adj[i]] == c) kc += a.L.w[i];
    const double tc = (c == cv) ? a.tot[c] - kv : a.tot[c];
    const double gain = kc - tc * kv / a.W;
    if (bc < 0 || better(gain, c, bg, bc, cv)) {
      bg = gain;
      bc = c;
    }
  }
  a.newcomm[v] = decide(a, cv, kv, a.tot[cv], a.csize[cv], bg, bc);
}

// One CTA per vertex; table in dynamic shared memory (slots = power of two) or,
// for the big bin, in global scratch at gtab_off[i].
template <bool GLOBAL_TABLE>
__global__ void __launch_bounds__(THREADS) k_move_cta(MoveArgs a, int slots) {
  extern __shared__ double s_dyn[];
  __shared__ double s_bg[THREADS / 32];
  __shared__ int s_bc[THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = blockIdx.x; i < a.nlist; i += gridDim.x) {
    const int v = a.list[i];
    const int b = a.L.off[v], e = a.L.off[v + 1];
    int nslots = slots;
    double* vals;
    int32_t* keys;
    if (GLOBAL_TABLE) {
      nslots = (int)(a.gtab_off[i + 1] - a.gtab_off[i]);
      vals = a.gtab_val + a.gtab_off[i];
      keys = a.gtab_key + a.gtab_off[i];
    } else {
      // table just large enough for this vertex (load factor <= 1/2), at most `slots`
      int need = 64;
      while (need < 2 * (e - b) && need < slots) need <<= 1;
      nslots = need;
      vals = s_dyn;
      keys = reinterpret_cast<int32_t*>(s_dyn + slots);
    }
    for (int s = threadIdx.x; s < nslots; s += THREADS) {
      keys[s] = EMPTY;
      vals[s] = 0.0;
    }
    __syncthreads();
    const int cv = a.comm[v];
    const double kv = a.kv[v];
    for (int j = b + threadIdx.x; j < e; j += THREADS)
      tab_add(keys, vals, (unsigned)nslots - 1u, a.comm[a.L.adj[j]], a.L.unit ? 1.0 : a.L.w[j]);
    __syncthreads();
    double bg = -INFINITY;
    int bc = -1;
    for (int s = threadIdx.x; s < nslots; s += THREADS) {
      const int c = keys[s];
      if (c != EMPTY) {
        const double tc = (c == cv) ? a.tot[c] - kv : a.tot[c];
        const double gain = vals[s] - tc * kv / a.W;
        if (bc < 0 || better(gain, c, bg, bc, cv)) {
          bg = gain;
          bc = c;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double og = __shfl_xor_sync(0xffffffffu, bg, o);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
      if (oc >= 0 && (bc < 0 || better(og, oc, bg, bc, cv))) {
        bg = og;
        bc = oc;
      }
    }
    if (lane == 0) {
      s_bg[wid] = bg;
      s_bc[wid] = bc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 1; k < THREADS / 32; ++k)
        if (s_bc[k] >= 0 && (bc < 0 || better(s_bg[k], s_bc[k], bg, bc, cv))) {
          bg = s_bg[k];
          bc = s_bc[k];
        }
      a.newcomm[v] = decide(a, cv, kv, a.tot[cv], a.csize[cv], bg, bc);
    }
    __syncthreads();
  }
}

__global__ void k_kv(Level L, double* kv, double* W) {
  const int lane = threadIdx.x & 31;
  double acc = 0;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < L.n; v += (gridDim.x * blockDim.x) >> 5) {
    double s = 0;
    for (int j = L.off[v] + lane; j < L.off[v + 1]; j += 32) s += L.unit ? 1.0 : L.w[j];
    s = warp_sum(s);
    if (lane == 0) {
      kv[v] = s + L.sl[v];
      acc += s + L.sl[v];
    }
  }
  if (W && lane == 0 && acc != 0.0) atomicAdd(W, acc);
}

__global__ void k_init_comm(int n, int32_t* comm, int32_t* newcomm) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) comm[v] = newcomm[v] = v;
}

__global__ void k_apply(int n, int parity, int32_t* comm, const int32_t* __restrict__ newcomm, int* moved) {
  int local = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if ((int)(hmix((unsigned)v) & 1u) != parity) continue;
    if (comm[v] != newcomm[v]) {
      comm[v] = newcomm[v];
      ++local;
    }
  }
  local = warp_sum(local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(moved, local);
}

// tot_c = sum of k_v and csize_c = members, per community. Lanes of a warp that hold
// the same community add up first (members of a community are mostly neighbours in
// the vertex order), so the hot communities see one atomic per group, not per vertex.
__global__ void k_tot(int n, const int32_t* __restrict__ comm, const double* __restrict__ kv, double* tot,
                      int32_t* csize) {
  const int lane = threadIdx.x & 31;
  const int n32 = (n + 31) & ~31;  // every lane of a warp runs the same iterations
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n32; v += gridDim.x * blockDim.x) {
    const bool on = v < n;
    const int c = on ? comm[v] : -1 - lane;  // idle lanes: keys no real community has
    const double k = on ? kv[v] : 0.0;
    const unsigned grp = __match_any_sync(0xffffffffu, c);
    double sum = 0.0;
    for (unsigned m = grp; m; m &= m - 1) sum += __shfl_sync(grp, k, __ffs(m) - 1);
    if (on && lane == __ffs(grp) - 1) {
      atomicAdd(&tot[c], sum);
      atomicAdd(&csize[c], __popc(grp));
    }
  }
}

// Q = sum_c in_c / W - (tot_c / W)^2 needs only the total internal weight
// sum_c in_c = sum_v (weight of v's edges inside its community + its self-loop):
// one partial per CTA, no per-community atomics; the host adds the partials of both
// kernels in CTA order, so Q is the same on every run. A warp takes 32 vertices at a
// time and spreads their edges over its lanes (an exclusive scan of the degrees), four
// 32-edge steps with their loads in flight together: the row walk of one vertex per
// warp was a chain of dependent loads per vertex (SBM 1M: 318 us per call).
__global__ void __launch_bounds__(THREADS) k_internal(Level L, const int32_t* __restrict__ comm, double W,
                                                      double* q) {
  constexpr int U = 4;
  __shared__ double s_red[THREADS / 32];
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double acc = 0;
  for (int base = gw * 32; base < L.n; base += nw * 32) {
    const int v = base + lane;
    int b = 0, d = 0, cv = -1;
    if (v < L.n) {
      b = L.off[v];
      d = L.off[v + 1] - b;
      cv = comm[v];
      acc += L.sl[v];
    }
    int inc = d;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, k);
      if (lane >= k) inc += t;
    }
    const int total = __shfl_sync(0xffffffffu, inc, 31);
    const int excl = inc - d;
    for (int t0 = 0; t0 < total; t0 += 32 * U) {
      int u[U], cq[U];
      double wq[U];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int t = t0 + 32 * q + lane;
        int j = 0;  // the last lane whose edges start at or before t
#pragma unroll
        for (int k = 16; k > 0; k >>= 1)
          if (__shfl_sync(0xffffffffu, excl, j + k) <= t) j += k;
        const int jb = __shfl_sync(0xffffffffu, b, j);
        const int je = __shfl_sync(0xffffffffu, excl, j);
        cq[q] = __shfl_sync(0xffffffffu, cv, j);
        u[q] = -1;
        wq[q] = 0.0;
        if (t < total) {
          const int k = jb + (t - je);
          u[q] = L.adj[k];
          wq[q] = L.unit ? 1.0 : L.w[k];
        }
      }
#pragma unroll
      for (int q = 0; q < U; ++q)
        if (u[q] >= 0 && comm[u[q]] == cq[q]) acc += wq[q];
    }
  }
  acc = block_sum<THREADS>(acc, s_red);
  if (threadIdx.x == 0) q[blockIdx.x] = acc / W;
}

__global__ void k_q(int n, const double* __restrict__ tot, double W, double* q) {
  __shared__ double s_red[THREADS / 32];
  double acc = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const double t = tot[c] / W;
    acc -= t * t;
  }
  acc = block_sum<THREADS>(acc, s_red);
  if (threadIdx.x == 0) q[blockIdx.x] = acc;
}

// ---- aggregation
__global__ void k_mark(int n, const int32_t* __restrict__ comm, int32_t* used) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) used[comm[v]] = 1;
}

__global__ void k_count_ext(Level L, const int32_t* __restrict__ comm, int32_t* cnt) {
  const int lane = threadIdx.x & 31;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < L.n; v += (gridDim.x * blockDim.x) >> 5) {
    const int cv = comm[v];
    int c = 0;
    for (int j = L.off[v] + lane; j < L.off[v + 1]; j += 32) c += comm[L.adj[j]] != cv;
    c = warp_sum(c);
    if (lane == 0) cnt[v] = c;
  }
}

// External edge (v, u) of the level -> key newid[comm v] * C + newid[comm u], at the
// scan position of v's external edges (in edge order)
__global__ void k_emit(Level L, const int32_t* __restrict__ comm, const int32_t* __restrict__ newid,
                       const int32_t* __restrict__ pos, unsigned long long C, unsigned long long* keys, double* vals,
                       double* sl_new) {
  const int lane = threadIdx.x & 31;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < L.n; v += (gridDim.x * blockDim.x) >> 5) {
    const int cv = comm[v];
    const unsigned long long nv = (unsigned long long)newid[cv];
    int base = pos[v];
    double inw = 0;
    for (int j0 = L.off[v]; j0 < L.off[v + 1]; j0 += 32) {
      const int j = j0 + lane;
      bool ext = false;
      int cu = 0;
      if (j < L.off[v + 1]) {
        cu = comm[L.adj[j]];
        ext = cu != cv;
        if (!ext) inw += L.w[j];
      }
      const unsigned m = __ballot_sync(0xffffffffu, ext);
      if (ext) {
        const int p = base + __popc(m & ((1u << lane) - 1u));
        keys[p] = nv * C + (unsigned long long)(unsigned)newid[cu];
        vals[p] = L.w[j];
      }
      base += __popc(m);
    }
    inw = warp_sum(inw);
    if (lane == 0 && (inw != 0.0 || L.sl[v] != 0.0)) atomicAdd(&sl_new[nv], inw + L.sl[v]);
  }
}

// One warp per run r of equal sorted keys [start[r], start[r + 1]): the next level's
// edge r (column key % C, weight = the run's sum: lane-strided partial sums, then a
// fixed xor tree) and one more edge in row key / C.
__global__ void k_merge_runs(int runs, const int32_t* __restrict__ start, const unsigned long long* __restrict__ keys,
                             const double* __restrict__ vals, unsigned long long C, int32_t* __restrict__ adj,
                             double* __restrict__ w, int32_t* __restrict__ rowcnt) {
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < runs; r += (gridDim.x * blockDim.x) >> 5) {
    const int b = start[r], e = start[r + 1];
    double acc = 0.0;
    for (int j = b + lane; j < e; j += 32) acc += vals[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      const unsigned long long k = keys[b];
      adj[r] = (int32_t)(k % C);
      w[r] = acc;
      atomicAdd(&rowcnt[(int)(k / C)], 1);
    }
  }
}

__global__ void k_compose(int n0, int32_t* orig, const int32_t* __restrict__ comm, const int32_t* __restrict__ newid) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n0; v += gridDim.x * blockDim.x) orig[v] = newid[comm[orig[v]]];
}

__global__ void k_f2d(const float* __restrict__ a, double* b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a ? (double)a[i] : 1.0;
}

// Vertex lists per (degree class, sub-sweep parity): list 2 * b + parity, b = 0 warp,
// 1 CTA, 2 CTA with a global table; each list holds at most cap entries.
// cta_deg: the CTA bin's bound, or sel[0] / 2 when the level's variant was chosen on the device
__global__ void k_bins(int n, const int32_t* __restrict__ off, int32_t* lists, int* counts, int cap, int cta_deg,
                       const int* __restrict__ sel) {
  if (sel) cta_deg = sel[0] / 2;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int d = off[v + 1] - off[v];
    const int b = d <= WARP_DEG ? 0 : (d <= cta_deg ? 1 : 2);
    const int k = 2 * b + (int)(hmix((unsigned)v) & 1u);
    const int p = atomicAdd(&counts[k], 1);
    lists[(size_t)k * cap + p] = v;
  }
}

}  // namespace lv

struct LvPlan {
  // level graphs (ping-pong)
  dbuf<int32_t> off[2], adj[2];
  dbuf<double> w[2], sl[2];
  dbuf<int32_t> comm, newcomm, csize, used, newid, cnt, pos, orig, lists, rowcnt;
  dbuf<double> kv, tot, scal, qpart;
  dbuf<unsigned long long> keys, skeys;
  dbuf<double> vals, svals;
  dbuf<int32_t> head, ridx, rstart, scr;
  dbuf<int> icnt;  // [0, 6) bin sizes, [6] moves applied, [8 ..) the level's variant (lv::SEL)
  dbuf<unsigned long long> vacc;  // the level's degree statistics
  dbuf<float> vmodel;             // the variant model on the device, generation vmodel_gen
  unsigned vmodel_gen = 0;
  dbuf<double> gval;
  dbuf<int32_t> gkey;
  dbuf<int64_t> goff;
};

void free_lv_plan(LvPlan* p) { delete p; }

namespace {

int dev_scan(LvPlan* p, const int32_t* in, int32_t* out, int n, cudaStream_t s) {
  SP_TRY(p->scr.alloc(prim::scan_scratch(n)));
  return prim::scan_exclusive<int32_t>(in, out, n, p->scr.p, s);
}

int read_int(const int* d, int* h, cudaStream_t s) { return copy_out(h, d, sizeof(int), s); }

}  // namespace

static int lv_modularity(LvPlan* p, const lv::Level& L, double W, cudaStream_t s, double* q) {
  const int n = L.n;
  const int g = num_sms() * 8;
  SP_TRY(p->qpart.alloc(2 * (size_t)g));
  lv::k_internal<<<g, lv::THREADS, 0, s>>>(L, p->comm.p, W, p->qpart.p);
  SP_CHECK_LAUNCH();
  lv::k_q<<<g, lv::THREADS, 0, s>>>(n, p->tot.p, W, p->qpart.p + g);
  SP_CHECK_LAUNCH();
  std::vector<double> part(2 * (size_t)g);
  SP_TRY(copy_out(part.data(), p->qpart.p, sizeof(double) * part.size(), s));
  double in = 0, sq = 0;
  for (int i = 0; i < g; ++i) in += part[i];
  for (int i = 0; i < g; ++i) sq += part[g + i];
  *q = in + sq;
  return SP_OK;
}

static int lv_recount(LvPlan* p, int n, cudaStream_t s) {
  SP_CHECK_CUDA(cudaMemsetAsync(p->tot.p, 0, sizeof(double) * n, s));
  SP_CHECK_CUDA(cudaMemsetAsync(p->csize.p, 0, sizeof(int32_t) * n, s));
  lv::k_tot<<<num_sms() * 8, 256, 0, s>>>(n, p->comm.p, p->kv.p, p->tot.p, p->csize.p);
  SP_CHECK_LAUNCH();
  return SP_OK;
}

// One sub-sweep over the vertices of one parity, all degree bins. counts[2 * b + parity]
// = entries of list (b, parity); the global tables of parity 1's big list follow
// parity 0's in gtab_off.
static int lv_subsweep(LvPlan* p, lv::MoveArgs a, const int counts[6], int cap, int parity, bool plain,
                       int slots, cudaStream_t s) {
  a.parity = parity;
  if (plain) {
    const int tb = 512;  // the generated code's launch shape (backend_cuda/dsl_cpp_generator.cpp:56-77)
    lv::k_move_plain<<<(a.L.n + tb - 1) / tb, tb, 0, s>>>(a);
    SP_CHECK_LAUNCH();
    return SP_OK;
  }
  const int g = num_sms() * 8;
  auto list = [&](int b) { return p->lists.p + (size_t)(2 * b + parity) * cap; };
  if (counts[0 + parity]) {
    a.list = list(0);
    a.nlist = counts[0 + parity];
    lv::k_move_warp<<<g, lv::THREADS, 0, s>>>(a);
    SP_CHECK_LAUNCH();
  }
  if (counts[2 + parity]) {
    a.list = list(1);
    a.nlist = counts[2 + parity];
    // degree <= slots / 2 fits at load factor <= 1/2; smaller tables fit more CTAs per SM
    const size_t dyn = (size_t)slots * (sizeof(double) + sizeof(int32_t));
    SP_CHECK_CUDA(cudaFuncSetAttribute(lv::k_move_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(lv::CTA_SLOTS_MAX * (sizeof(double) + sizeof(int32_t)))));
    int per_sm = 1;
    SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lv::k_move_cta<false>, lv::THREADS, dyn));
    lv::k_move_cta<false><<<num_sms() * std::max(1, per_sm), lv::THREADS, dyn, s>>>(a, slots);
    SP_CHECK_LAUNCH();
  }
  if (counts[4 + parity]) {
    a.list = list(2);
    a.nlist = counts[4 + parity];
    a.gtab_off = p->goff.p + (parity ? counts[4] : 0);
    lv::k_move_cta<true><<<num_sms() * 2, lv::THREADS, 0, s>>>(a, 0);
    SP_CHECK_LAUNCH();
  }
  return SP_OK;
}

// ---- learned kernel variant, per level ---------------------------------------------
// The shared-memory table of the CTA bin: vertices above WARP_DEG and up to slots / 2
// edges get a CTA with a table of slots entries in shared memory (smaller tables fit more
// CTAs per SM); longer rows use tables in global memory. The last entry is the fixed
// default. The choice is made on the device: the level's degree statistics, the inputs
// of every candidate and the network's scores never leave it, and the degree bins read
// the chosen bound there.
namespace lv {
constexpr int VSLOTS[] = {1024, 2048, 4096, 8192, CTA_SLOTS_MAX};
constexpr int N_VARIANTS = (int)(sizeof(VSLOTS) / sizeof(VSLOTS[0]));
constexpr int DEFAULT_VARIANT = N_VARIANTS - 1;
// degree thresholds of the level statistics: WARP_DEG, then slots / 2 of each candidate
constexpr int VTHR[6] = {WARP_DEG, 512, 1024, 2048, 4096, CTA_SLOTS_MAX / 2};
static_assert(N_VARIANTS + 1 == 6, "one threshold per candidate after WARP_DEG");
constexpr int SEL = 8;  // icnt[SEL]: chosen slots, [SEL + 1] candidate, [SEL + 2 ..] its inputs (float bits)

__host__ __device__ inline int vslots(int cand) { return 1024 << cand; }  // = VSLOTS[cand]

// Inputs of candidate cand on a level graph of n vertices and m entries, from its degree
// statistics acc (thresholds VTHR, layout of degree_stats_launch): the level's shape, the
// level index, the share of entries and the rows above WARP_DEG, then the candidate's
// table size, the entries in its shared-table and global-table bins, and the rows of each.
__host__ __device__ inline void level_features(int n, double m, int level, const unsigned long long* acc, int cand,
                                               float* x) {
  const int t = cand + 1;  // VTHR[t] = slots / 2
  const double N = n > 1 ? (double)n : 1.0, M = m > 1.0 ? m : 1.0;
  const double r0 = (double)acc[2], e0 = (double)acc[3], rt = (double)acc[2 + 2 * t], et = (double)acc[3 + 2 * t];
  x[0] = (float)log2(N);
  x[1] = (float)log2(M + 1.0);
  x[2] = (float)(M / N);
  x[3] = (float)log2((double)acc[0] + 1.0);
  x[4] = (float)log2((double)acc[1] / M + 1.0);
  x[5] = (float)level;
  x[6] = (float)(e0 / M);
  x[7] = (float)log2(r0 + 1.0);
  x[8] = (float)log2((double)vslots(cand));
  x[9] = (float)((e0 - et) / M);
  x[10] = (float)(et / M);
  x[11] = (float)log2(rt + 1.0);
  x[12] = (float)log2((r0 - rt) + 1.0);
}

// One CTA of N_VARIANTS * 32 threads: the inputs of every candidate, then the candidate
// (forced >= 0; else the network's lowest score with the margin rule toward dflt when a
// model is given; else dflt), its slots and its inputs into sel.
__global__ void __launch_bounds__(N_VARIANTS * 32) k_choose(const unsigned long long* __restrict__ acc,
                                                            const int32_t* __restrict__ off, int n, int level,
                                                            const float* __restrict__ model, int forced, int dflt,
                                                            int* sel) {
  __shared__ float rows[N_VARIANTS][SP_MLP_IN];
  __shared__ float raw[N_VARIANTS][SP_MLP_IN];
  const int t = threadIdx.x;
  if (t < N_VARIANTS) {
    level_features(n, (double)off[n], level, acc, t, raw[t]);
    for (int i = 0; i < SP_MLP_IN; ++i) rows[t][i] = raw[t][i];
  }
  int cand = forced >= 0 ? forced : dflt;
  if (model && forced < 0) {
    cand = mlp_argmin<N_VARIANTS>(model, rows, 0, dflt, model[SP_MLP_PARAMS + 2 * SP_MLP_IN]);
  } else {
    __syncthreads();
  }
  if (t == 0) {
    sel[0] = vslots(cand);
    sel[1] = cand;
  }
  if (t < SP_MLP_IN) sel[2 + t] = __float_as_int(raw[cand][t]);
}
}  // namespace lv

int lv_variant_count() { return lv::N_VARIANTS; }

int lv_variant_features(sp_graph* g, int cand, float* x, int* applicable) {
  if (cand < 0 || cand >= lv::N_VARIANTS) return SP_ERR_INVALID;
  DegStats ds;
  SP_TRY(degree_stats(g->off.p, g->V, lv::VTHR, 6, g->stream, &ds));
  unsigned long long acc[2 + 2 * DEG_THR_MAX] = {};
  acc[0] = (unsigned long long)ds.max_deg;
  acc[1] = (unsigned long long)ds.sum_sq;
  for (int i = 0; i < 6; ++i) {
    acc[2 + 2 * i] = (unsigned long long)ds.rows_above[i];
    acc[3 + 2 * i] = (unsigned long long)ds.edges_above[i];
  }
  lv::level_features(g->V, (double)g->E, 0, acc, cand, x);
  *applicable = 1;
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_louvain(sp_graph_h g, const float* weight, double threshold, int32_t* community, double* modularity,
                          int32_t* levels_out, int32_t* sweeps_out, int32_t variant) {
  int total_sweeps = 0;
  if (!g || !modularity) {
    set_error("sp_louvain: invalid argument");
    return SP_ERR_INVALID;
  }
  if (variant != SP_LV_TUNED && variant != SP_LV_PLAIN) {
    set_error("sp_louvain: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  const bool plain = variant == SP_LV_PLAIN;
  if (!plain) g->lv_trace_rec.clear();
  if (!g->lv) g->lv = new LvPlan();
  LvPlan* p = g->lv;
  cudaStream_t s = g->stream;
  const int n0 = g->V;
  const int64_t m0 = g->E;
  const int gs = num_sms() * 8;
  // level 0 = the input graph; weights as FP64
  SP_TRY(p->off[0].alloc(n0 + 1));
  SP_TRY(p->adj[0].alloc(m0));
  SP_TRY(p->w[0].alloc(m0));
  SP_TRY(p->sl[0].alloc(n0));
  SP_CHECK_CUDA(cudaMemcpyAsync(p->off[0].p, g->off.p, sizeof(int32_t) * (n0 + 1), cudaMemcpyDeviceToDevice, s));
  if (m0) SP_CHECK_CUDA(cudaMemcpyAsync(p->adj[0].p, g->adj.p, sizeof(int32_t) * m0, cudaMemcpyDeviceToDevice, s));
  const float* dw = nullptr;
  dbuf<float> wtmp;
  if (weight) {
    SP_TRY(wtmp.alloc(m0));
    if (m0) SP_CHECK_CUDA(cudaMemcpyAsync(wtmp.p, weight, sizeof(float) * m0, cudaMemcpyDefault, s));
    dw = wtmp.p;
  }
  lv::k_f2d<<<gs, 256, 0, s>>>(dw, p->w[0].p, m0);
  SP_CHECK_LAUNCH();
  SP_CHECK_CUDA(cudaMemsetAsync(p->sl[0].p, 0, sizeof(double) * n0, s));
  SP_TRY(p->comm.alloc(n0));
  SP_TRY(p->newcomm.alloc(n0));
  SP_TRY(p->csize.alloc(n0));
  SP_TRY(p->used.alloc(n0 + 1));
  SP_TRY(p->newid.alloc(n0 + 1));
  SP_TRY(p->cnt.alloc(n0 + 1));
  SP_TRY(p->pos.alloc(n0 + 1));
  SP_TRY(p->orig.alloc(n0));
  SP_TRY(p->lists.alloc((size_t)6 * n0));
  SP_TRY(p->rowcnt.alloc(n0 + 1));
  SP_TRY(p->kv.alloc(n0));
  SP_TRY(p->tot.alloc(n0));
  SP_TRY(p->scal.alloc(2));
  SP_TRY(p->icnt.alloc(32));
  lv::k_init_comm<<<gs, 256, 0, s>>>(n0, p->orig.p, p->newcomm.p);  // orig[v] = v
  SP_CHECK_LAUNCH();

  // total weight W (constant over levels)
  // unweighted input: level 0's weights are all 1.0 and the kernels do not read them
  lv::Level L{n0, p->off[0].p, p->adj[0].p, p->w[0].p, p->sl[0].p, weight ? 0 : 1};
  SP_CHECK_CUDA(cudaMemsetAsync(p->scal.p + 1, 0, sizeof(double), s));
  lv::k_kv<<<gs, 256, 0, s>>>(L, p->kv.p, p->scal.p + 1);
  SP_CHECK_LAUNCH();
  double W = 0;
  SP_TRY(copy_out(&W, p->scal.p + 1, sizeof(double), s));
  if (!(W > 0)) {
    *modularity = 0.0;
    if (levels_out) *levels_out = 0;
    if (sweeps_out) *sweeps_out = 0;
    if (community) {
      lv::k_init_comm<<<gs, 256, 0, s>>>(n0, p->comm.p, p->newcomm.p);
      SP_CHECK_LAUNCH();
      SP_TRY(copy_out(community, p->comm.p, sizeof(int32_t) * n0, s));
    }
    return SP_OK;
  }

  int cur = 0, levels = 0;
  double qcur = 0;
  const int max_levels = 32, max_sweeps = 100;
  bool first = true;
  while (true) {
    const int n = L.n;
    // communities start as singletons
    lv::k_init_comm<<<gs, 256, 0, s>>>(n, p->comm.p, p->newcomm.p);
    SP_CHECK_LAUNCH();
    if (!first) {
      lv::k_kv<<<gs, 256, 0, s>>>(L, p->kv.p, nullptr);
      SP_CHECK_LAUNCH();
    }
    SP_TRY(lv_recount(p, n, s));
    double qlev0 = 0;
    SP_TRY(lv_modularity(p, L, W, s, &qlev0));
    if (first) qcur = qlev0;
    first = false;
    // kernel variant of this level, chosen on the device (forced, learned, or the
    // defaults' inputs for the trace), then the degree bins
    const int mode = g->variant[VAR_LV];
    const int fixed_slots = g->lv_cta_slots > 0 ? g->lv_cta_slots : lv::CTA_SLOTS_MAX;
    unsigned gen = 0;
    if (!plain && mode == -1 && g->lv_cta_slots < 0) {
      std::vector<float> packed;
      gen = variant_model(VAR_LV, packed);
      if (gen && p->vmodel_gen != gen) {
        SP_TRY(p->vmodel.alloc(packed.size()));
        SP_CHECK_CUDA(cudaMemcpyAsync(p->vmodel.p, packed.data(), sizeof(float) * packed.size(),
                                      cudaMemcpyHostToDevice, s));
        p->vmodel_gen = gen;
      }
    }
    const bool dev_sel = !plain && (mode >= 0 || gen || g->lv_trace);
    // trace: the level's choice, bins, tables and sweeps on the device clock
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (g->lv_trace && !plain) {
      SP_CHECK_CUDA(cudaEventCreate(&ev0));
      SP_CHECK_CUDA(cudaEventCreate(&ev1));
      SP_CHECK_CUDA(cudaEventRecord(ev0, s));
    }
    int* sel = p->icnt.p + lv::SEL;
    if (dev_sel) {
      int dflt = lv::DEFAULT_VARIANT;
      for (int k = 0; k < lv::N_VARIANTS; ++k)
        if (lv::VSLOTS[k] == fixed_slots) dflt = k;
      SP_TRY(p->vacc.alloc(2 + 2 * DEG_THR_MAX));
      SP_TRY(degree_stats_launch(L.off, n, lv::VTHR, 6, p->vacc.p, s));
      lv::k_choose<<<1, lv::N_VARIANTS * 32, 0, s>>>(p->vacc.p, L.off, n, levels, gen ? p->vmodel.p : nullptr,
                                                      mode >= 0 ? mode : -1, dflt, sel);
      SP_CHECK_LAUNCH();
    }
    SP_CHECK_CUDA(cudaMemsetAsync(p->icnt.p, 0, sizeof(int) * 6, s));
    lv::k_bins<<<gs, 256, 0, s>>>(n, L.off, p->lists.p, p->icnt.p, n0, fixed_slots / 2, dev_sel ? sel : nullptr);
    SP_CHECK_LAUNCH();
    int hsel[lv::SEL + 2 + SP_MLP_IN];
    SP_TRY(copy_out(hsel, p->icnt.p, sizeof(int) * (dev_sel ? lv::SEL + 2 + SP_MLP_IN : 6), s));
    int counts[6];
    for (int k = 0; k < 6; ++k) counts[k] = hsel[k];
    const int slots = dev_sel ? hsel[lv::SEL] : fixed_slots;
    const int lcand = dev_sel && (mode >= 0 || gen) ? hsel[lv::SEL + 1] : -1;
    g->last_variant[VAR_LV] = lcand;
    const int nbig = counts[4] + counts[5];
    if (nbig && !plain) {
      // global tables for the highest-degree vertices (both parities' lists, in that
      // order): 2 * degree slots, a power of two
      std::vector<int32_t> big(nbig);
      if (counts[4]) SP_TRY(copy_out(big.data(), p->lists.p + 4 * (size_t)n0, sizeof(int32_t) * counts[4], s));
      if (counts[5])
        SP_TRY(copy_out(big.data() + counts[4], p->lists.p + 5 * (size_t)n0, sizeof(int32_t) * counts[5], s));
      std::vector<int32_t> hoff(n + 1);
      SP_TRY(copy_out(hoff.data(), L.off, sizeof(int32_t) * (n + 1), s));
      std::vector<int64_t> go(nbig + 1, 0);
      for (int k = 0; k < nbig; ++k) {
        int64_t d = hoff[big[k] + 1] - hoff[big[k]], sl = 1;
        while (sl < 2 * d) sl <<= 1;
        go[k + 1] = go[k] + sl;
      }
      SP_TRY(p->goff.alloc(nbig + 1));
      SP_TRY(p->gval.alloc(go.back()));
      SP_TRY(p->gkey.alloc(go.back()));
      SP_CHECK_CUDA(cudaMemcpyAsync(p->goff.p, go.data(), sizeof(int64_t) * go.size(), cudaMemcpyHostToDevice, s));
    }
    lv::MoveArgs a;
    a.L = L;
    a.comm = p->comm.p;
    a.tot = p->tot.p;
    a.csize = p->csize.p;
    a.kv = p->kv.p;
    a.newcomm = p->newcomm.p;
    a.W = W;
    a.gtab_val = p->gval.p;
    a.gtab_key = p->gkey.p;
    a.gtab_off = p->goff.p;
    double qold = qlev0, qnew = qlev0;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
      for (int parity = 0; parity < 2; ++parity) {
        SP_TRY(lv_subsweep(p, a, counts, n0, parity, plain, slots, s));
        SP_CHECK_CUDA(cudaMemsetAsync(p->icnt.p + 6, 0, sizeof(int), s));
        lv::k_apply<<<gs, 256, 0, s>>>(n, parity, p->comm.p, p->newcomm.p, p->icnt.p + 6);
        SP_CHECK_LAUNCH();
        SP_TRY(lv_recount(p, n, s));
      }
      qold = qnew;
      ++total_sweeps;
      SP_TRY(lv_modularity(p, L, W, s, &qnew));
      if (!(qnew - qold > threshold)) break;
    }
    if (ev0) {
      // trace record: the inputs of the variant that ran, its index, the level's sweep
      // loop in device milliseconds
      float ms = 0;
      SP_CHECK_CUDA(cudaEventRecord(ev1, s));
      SP_CHECK_CUDA(cudaEventSynchronize(ev1));
      SP_CHECK_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      cudaEventDestroy(ev0);
      cudaEventDestroy(ev1);
      std::vector<float>& tr = g->lv_trace_rec;
      float lx[SP_MLP_IN];
      memcpy(lx, hsel + lv::SEL + 2, sizeof(lx));
      tr.insert(tr.end(), lx, lx + SP_MLP_IN);
      tr.push_back((float)hsel[lv::SEL + 1]);
      tr.push_back(ms);
      tr.push_back(0.0f);
    }
    ++levels;
    // renumber communities
    SP_CHECK_CUDA(cudaMemsetAsync(p->used.p, 0, sizeof(int32_t) * (n + 1), s));
    lv::k_mark<<<gs, 256, 0, s>>>(n, p->comm.p, p->used.p);
    SP_CHECK_LAUNCH();
    SP_TRY(dev_scan(p, p->used.p, p->newid.p, n + 1, s));
    int C = 0;
    SP_TRY(copy_out(&C, p->newid.p + n, sizeof(int32_t), s));
    lv::k_compose<<<gs, 256, 0, s>>>(n0, p->orig.p, p->comm.p, p->newid.p);
    SP_CHECK_LAUNCH();
    const bool improved = qnew - qcur > threshold;
    qcur = std::max(qcur, qnew);
    if (!improved || C == n || levels >= max_levels) {
      qcur = qnew;
      break;
    }
    // aggregate: communities become vertices
    const int nx = cur ^ 1;
    lv::k_count_ext<<<gs, 256, 0, s>>>(L, p->comm.p, p->cnt.p);
    SP_CHECK_LAUNCH();
    SP_CHECK_CUDA(cudaMemsetAsync(p->cnt.p + n, 0, sizeof(int32_t), s));
    SP_TRY(dev_scan(p, p->cnt.p, p->pos.p, n + 1, s));
    int mx = 0;
    SP_TRY(copy_out(&mx, p->pos.p + n, sizeof(int32_t), s));
    SP_TRY(p->keys.alloc(std::max(1, mx)));
    SP_TRY(p->vals.alloc(std::max(1, mx)));
    SP_TRY(p->skeys.alloc(std::max(1, mx)));
    SP_TRY(p->svals.alloc(std::max(1, mx)));
    SP_TRY(p->sl[nx].alloc(C));
    SP_CHECK_CUDA(cudaMemsetAsync(p->sl[nx].p, 0, sizeof(double) * C, s));
    const unsigned long long CC = (unsigned long long)C;
    lv::k_emit<<<gs, 256, 0, s>>>(L, p->comm.p, p->newid.p, p->pos.p, CC, p->keys.p, p->vals.p, p->sl[nx].p);
    SP_CHECK_LAUNCH();
    int key_bits = 1;  // keys are below C * C
    while (key_bits < 63 && (1ull << key_bits) < CC * CC) ++key_bits;
    SP_TRY(p->scr.alloc(std::max(prim::sort_scratch(mx), prim::scan_scratch((int64_t)mx + 1))));
    unsigned long long* sk = nullptr;
    double* sv = nullptr;
    SP_TRY(prim::radix_sort_pairs(p->keys.p, p->vals.p, p->skeys.p, p->svals.p, mx, key_bits, p->scr.p, &sk, &sv, s));
    // runs of equal keys: heads, their scan, run starts
    SP_TRY(p->head.alloc((size_t)mx + 1));
    SP_TRY(p->ridx.alloc((size_t)mx + 1));
    prim::k_run_heads<<<gs, 256, 0, s>>>(sk, mx, p->head.p);
    SP_CHECK_LAUNCH();
    SP_TRY(prim::scan_exclusive<int32_t>(p->head.p, p->ridx.p, (int64_t)mx + 1, p->scr.p, s));
    int mu = 0;
    SP_TRY(read_int(p->ridx.p + mx, &mu, s));
    SP_TRY(p->rstart.alloc((size_t)mu + 1));
    prim::k_run_starts<<<gs, 256, 0, s>>>(p->head.p, p->ridx.p, mx, p->rstart.p);
    SP_CHECK_LAUNCH();
    g_launches += 2;
    SP_TRY(p->off[nx].alloc(C + 1));
    SP_TRY(p->adj[nx].alloc(std::max(1, mu)));
    SP_TRY(p->w[nx].alloc(std::max(1, mu)));
    SP_CHECK_CUDA(cudaMemsetAsync(p->rowcnt.p, 0, sizeof(int32_t) * (C + 1), s));
    if (mu) {
      lv::k_merge_runs<<<gs, 256, 0, s>>>(mu, p->rstart.p, sk, sv, CC, p->adj[nx].p, p->w[nx].p, p->rowcnt.p);
      SP_CHECK_LAUNCH();
      g_launches++;
    }
    SP_TRY(dev_scan(p, p->rowcnt.p, p->off[nx].p, C + 1, s));
    cur = nx;
    L = lv::Level{C, p->off[cur].p, p->adj[cur].p, p->w[cur].p, p->sl[cur].p, 0};
  }
  *modularity = qcur;
  if (levels_out) *levels_out = levels;
  if (sweeps_out) *sweeps_out = total_sweeps;
  if (community) SP_TRY(copy_out(community, p->orig.p, sizeof(int32_t) * n0, s));
  return SP_OK;
}

extern "C" int sp_louvain_level_trace(sp_graph_h g, float* records, int32_t cap, int32_t* n) {
  if (!g || !n || cap < 0 || (cap > 0 && !records)) {
    set_error("sp_louvain_level_trace: invalid argument");
    return SP_ERR_INVALID;
  }
  const int k = (int)(g->lv_trace_rec.size() / 16);
  *n = k;
  const int c = std::min(k, (int)cap);
  if (c) memcpy(records, g->lv_trace_rec.data(), sizeof(float) * 16 * (size_t)c);
  return SP_OK;
}
