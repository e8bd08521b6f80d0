// Single-source shortest paths for sm_100a.
//
// Semantics: DSL staticDSLCodes/sssp_dslV3:1-26 — the reference's fixed point
// (backend_omp/dsl_cpp_generator.cpp:2637-2708, Min reduction :297-527; CUDA
// atomicMin :679-825) converges to exact shortest-path distances; unreachable
// vertices keep INT_MAX (:1993-2025). Any correct SSSP gives bit-identical int32
// distances, which is what the parity tests require.
//
// SP_SSSP_DELTA: delta-stepping in ONE persistent cooperative kernel (no host
// round trips), with bounded grid barriers (sp_sync.cuh):
//   * near queue Q (ping-pong) holds vertices whose distance dropped below the
//     current bucket threshold; far pile F holds the rest;
//   * relax rounds: every frontier vertex pushes along its out-edges with
//     atomicMin. A warp holds up to 32 frontier vertices, one per lane, and their
//     edges are flattened over its lanes (an exclusive scan of the degrees), 32
//     edges per step, so a 4-neighbour grid vertex costs one step, not four; a
//     small frontier is spread over all warps. SU steps go together: their dist
//     loads, atomicMins and mark updates are all issued before any is waited
//     for, and their queue appends share one counter atomic. Vertices above hub_deg out-edges
//     (R-MAT hubs) are queued in a hub list whose chunks all warps share in the
//     next round; queue appends are warp-aggregated and de-duplicated with
//     per-round / per-epoch mark bitmaps;
//   * warp-local cascades (rounds whose frontier is at most 32 vertices per warp):
//     a vertex a warp improves below the bucket threshold goes to the warp's ring
//     in shared memory instead of the next round's queue, and the warp relaxes its
//     ring until it is empty or its edge budget (sssp.local warp steps) is spent,
//     then moves what is left to the queue. On a high-diameter graph one round then
//     covers many hops of the same bucket, where each hop used to cost a grid
//     barrier. Ring entries carry no mark: every improvement puts its vertex in
//     the ring (or, when full, in the marked queue), so the last improvement of a
//     vertex is always relaxed after it;
//   * when Q empties, the threshold jumps to the bucket of the smallest far
//     distance and F is split into Q and the next far pile.
//   Negative weights switch to delta = infinity (queue-based Bellman-Ford), bounded
//   by V rounds (a longer run means a negative cycle).
// SP_SSSP_PLAIN: the generated CUDA form — one thread per vertex over all V each
// iteration, modified flags, atomicMin, host loop on a finished flag.
#include <climits>
#include <cmath>
#include <vector>

#include "sp_internal.cuh"
#include "sp_mlp_dev.cuh"
#include "sp_sync.cuh"

namespace sp {

namespace ss {
constexpr int THREADS = 256;
// Queued vertices above HUB_DEG out-edges are relaxed in HUB_CHUNK-edge pieces that
// every warp shares, so no warp walks a long row alone while the others wait at the
// round's barrier. R-MAT 23 (learned schedule): 12.6 ms at (2048, 256), 11.5 at
// (512, 128), 11.2 at (128, 64), 12.0 at (32, 32).
constexpr int HUB_DEG = 128;
constexpr int HUB_CHUNK = 64;
constexpr int HUB_DEG_MAX = 1 << 25;  // 32 entries of at most this degree sum below 2^31
constexpr int RING = 256;             // entries of a warp's cascade ring (power of two)
constexpr int LOCAL_STEPS = 64;       // default cascade budget: 32-edge warp steps per round
constexpr int SU = 4;                 // 32-edge steps whose loads and atomics are in flight together
// Sources per cooperative launch of the batched form. 16 weighted closeness sources of
// undirected R-MAT 20: 34.1 ms with 1 per launch, 34.5 with 4 or 8, 36.0 with 16.
constexpr int BATCH = 4;
// sp_sssp_dynamic repairs a batch with deletions by default when the graph's last solve
// took at least this many rounds (grid 1024^2 repairs in 1.5 ms against 8.3 ms for a new
// solve; R-MAT 20, a dozen rounds, 3.4 against 2.2 ms).
constexpr int REPAIR_MIN_ROUNDS = 32;
constexpr unsigned FULL = 0xffffffffu;

struct Ctl {
  GridBar bar;
  int qcount[3];   // per round (mod 3): entries appended to the queue read next round
  unsigned long long hcount[3];  // per round (mod 3): (hub entries << 32) | hub chunks
  int fcount[3];   // per epoch (mod 3)
  int fmin[3];     // per epoch: smallest distance pushed to the far pile
  int rounds;      // relax rounds executed
  int epochs;
  int status;      // 0 ok, 1 timeout / round cap, 2 negative cycle suspected, 3 a buffer overflowed
  int pad;
  unsigned long long relaxed;  // edges relaxed over the run (work inflation = relaxed / E_r)
};

struct Args {
  const int32_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  const int32_t* __restrict__ w;
  int32_t* dist;
  int32_t* q[2];
  int32_t* f[2];
  int32_t* hv[2];      // hub vertices per round (ping-pong)
  int32_t* hbase[2];   // first chunk index of each hub entry (increasing)
  // Marks (one bit per vertex, 4 * nwords words): qbits(k) = bits + k * nwords says a
  // vertex is queued for a round of parity k, fbits(k) = bits + (2 + k) * nwords that it
  // is in the far pile of an epoch of parity k. Every phase clears the generation that no
  // phase of its own touches (k_delta's phases), so each bitmap is zero before its first
  // mark. At V = 2^23 they take 4 MB where two int32 stamp arrays took 67 MB of L2.
  unsigned* bits;
  int nwords;
  Ctl* ctl;
  int V;
  long long delta;      // bucket width; >= INT_MAX means a single bucket
  long long max_rounds;
  int hub_deg;          // vertices with more out-edges are relaxed in pieces by all warps
  int hub_chunk;        // edges per piece
  int local_edges;      // cascade budget of a warp per round, in edges (0 = no cascades)
  int filter;           // 1: load dist[u] and send the atomicMin only when it would lower it;
                        // 0: send the atomicMin straight away (one L2 round trip less per hop);
                        // -1: 0 in cascades, 1 elsewhere
  // Bucket width per epoch (the learned scheduler's per-iteration decision): 0 = every
  // bucket `delta` wide; 1 = the width factor whose predicted cost per unit of distance
  // advanced is lowest under the epoch model; 2 = a pseudo-random factor per epoch
  // (exploration, to collect training data).
  int epolicy;
  int ewiden;            // 1: only factors >= 1 (never narrower than the call's delta)
  unsigned eseed;
  const float* emodel;   // [SP_MLP_PARAMS + 2 * SP_MLP_IN]: parameters, feature mean, feature scale
  float* etrace;         // [etrace_cap][ETRACE]: per epoch, the chosen candidate's inputs, factor, advance
  unsigned long long* etime;  // [etrace_cap + 1]: globaltimer at each advance, then at the end
  int etrace_cap;
  float sfeat[4];        // log2 V, log2 E, mean out-degree, log2 largest weight
};

// Width factors of the per-epoch choice, as num / 4 of the call's delta.
constexpr int NFAC = 6;
__device__ __constant__ int kFacNum[NFAC] = {1, 2, 4, 8, 16, 32};
constexpr int ETRACE = 16;  // floats per trace record: SP_MLP_IN inputs, factor, advance, pad

// Where a round's relaxations go: the next round's queue and hub list, this
// epoch's far pile.
struct Out {
  int32_t* QN;
  int* qnext;
  int32_t* HV;
  int32_t* HB;
  unsigned long long* hnext;
  int32_t* F;
  int* fcnt;
  int* fmin;
};

// A warp's cascade ring in shared memory; head and cnt are warp-uniform.
struct Ring {
  int32_t* s;
  int head;
  int cnt;
};

// Adjacency and weights are streamed: each is read once per expansion of its vertex,
// so their loads skip L1 and are marked first to leave L2, which keeps dist, the
// mark bitmaps and the offsets (random accesses) resident. R-MAT 23: 9.1 -> 7.3 ms; grid
// 4096^2: 33.3 -> 33.8 ms. Marking the dist loads evict-last on top gained nothing.
__device__ __forceinline__ int ld_stream(const int32_t* p) {
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  int v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

// Sets vertex u's bit in bm; true for the one caller that set it first.
__device__ __forceinline__ bool mark(unsigned* bm, int u) {
  const unsigned b = 1u << (u & 31);
  return (atomicOr(bm + (u >> 5), b) & b) == 0u;
}
__device__ __forceinline__ unsigned* qbits(const Args& a, int round) { return a.bits + (size_t)(round & 1) * a.nwords; }
__device__ __forceinline__ unsigned* fbits(const Args& a, int epoch) {
  return a.bits + (size_t)(2 + (epoch & 1)) * a.nwords;
}

// A queue, hub list or far pile holds at most V entries (the marks admit each vertex
// once per round or epoch); an append past that is dropped and flagged (status 3), so
// a broken mark could never write outside the buffer.
__device__ __forceinline__ void put(const Args& a, int32_t* buf, int idx, int val) {
  if (idx < a.V)
    buf[idx] = val;
  else
    atomicExch(&a.ctl->status, 3);
}

// Warp-aggregated append of `want` lanes into buf via counter.
__device__ __forceinline__ void warp_push(const Args& a, bool want, int val, int32_t* buf, int* counter) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (want) put(a, buf, base + __popc(m & ((1u << lane) - 1u)), val);
}

// Queue u for the next round: hubs go to the hub list (with their chunk count),
// everything else to the near queue (warp-aggregated).
__device__ __forceinline__ void queue_push(const Args& a, bool want, int u, int32_t* QN, int* qnext, int32_t* HV,
                                           int32_t* HB, unsigned long long* hcnt) {
  bool hub = false;
  int nch = 0;
  if (want) {
    const int d = a.off[u + 1] - a.off[u];
    if (d > a.hub_deg) {
      hub = true;
      nch = (d + a.hub_chunk - 1) / a.hub_chunk;
    }
  }
  if (hub) {
    const unsigned long long old = atomicAdd(hcnt, (1ull << 32) | (unsigned long long)nch);
    const int idx = (int)(old >> 32);
    put(a, HV, idx, u);
    put(a, HB, idx, (int)(old & 0xffffffffull));
  }
  warp_push(a, want && !hub, u, QN, qnext);
}

// Below-threshold improvements of this step (want lanes). LOCAL: into the warp's
// ring while it has room, the rest marked into the next round's queue. Otherwise
// the caller's relax already marked them: straight into the queue.
template <bool LOCAL>
__device__ __forceinline__ void push_near(const Args& a, bool want, int u, int round, const Out& o, Ring& r) {
  if (LOCAL) {
    const unsigned m = __ballot_sync(FULL, want);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int room = RING - r.cnt;
    const int rank = __popc(m & ((1u << lane) - 1u));
    const bool mine = want && rank < room;
    if (mine) r.s[(r.head + r.cnt + rank) & (RING - 1)] = u;
    r.cnt += min(__popc(m), room);
    want = want && !mine && mark(qbits(a, round + 1), u);
  }
  queue_push(a, want, u, o.QN, o.qnext, o.HV, o.HB, o.hnext);
}

// Relax N edges per lane (nd = dist + weight for target u; nd >= INT_MAX: no edge):
// every dist load is issued, then every atomicMin, then every mark update, before
// any result is waited for. res: 1 = improved below the bucket threshold (with
// STAMP, only the first such improvement of u this round), 2 = improved above it
// and first in the far pile this epoch, 0 = nothing to queue. When two edges of a
// group hit the same vertex, the atomics decide; the loads only filter. The dist
// loads are skipped (every candidate goes to atomicMin) when a.filter is 0, and by
// default in cascades (!STAMP), where they would add a round trip to each hop: grid
// 4096^2 33.5 -> 30.6 ms; R-MAT 23 (no cascades) keeps them, where skipping them
// everywhere measured 6.6 against 6.4 ms. Carrying each ring entry's CSR row, loaded
// beside the atomicMin, to save the offset load of the next hop measured slower
// (33.6 ms on the grid).
template <bool STAMP, int N>
__device__ __forceinline__ void relax_group(const Args& a, const int (&u)[N], const long long (&nd)[N],
                                            long long thr, int round, int epoch, int* fmin_slot, int (&res)[N]) {
  const bool filt = a.filter < 0 ? STAMP : a.filter != 0;
  int cur[N], old[N];
#pragma unroll
  for (int q = 0; q < N; ++q)
    cur[q] = nd[q] < (long long)INT_MAX ? (filt ? __ldcg(a.dist + u[q]) : INT_MAX) : INT_MIN;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    old[q] = INT_MIN;
    if ((int)nd[q] < cur[q]) old[q] = atomicMin(a.dist + u[q], (int)nd[q]);
  }
#pragma unroll
  for (int q = 0; q < N; ++q) {
    res[q] = 0;
    const int ndi = (int)nd[q];
    if (ndi < old[q]) {
      if (nd[q] < thr) {
        res[q] = (!STAMP || mark(qbits(a, round + 1), u[q])) ? 1 : 0;
      } else {
        atomicMin(fmin_slot, ndi);
        res[q] = mark(fbits(a, epoch), u[q]) ? 2 : 0;
      }
    }
  }
}

// Appends the flagged values of N steps to buf with one counter atomic per warp.
template <int N>
__device__ __forceinline__ void warp_push_many(const Args& a, const bool (&want)[N], const int (&val)[N], int32_t* buf,
                                               int* counter) {
  unsigned m[N];
  int n = 0;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    m[q] = __ballot_sync(FULL, want[q]);
    n += __popc(m[q]);
  }
  if (n == 0) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0) base = atomicAdd(counter, n);
  base = __shfl_sync(FULL, base, 0);
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    if (want[q]) put(a, buf, base + __popc(m[q] & lt), val[q]);
    base += __popc(m[q]);
  }
}

// Next round's queue for N steps: vertices above hub_deg out-edges go to the hub list
// (their degree loads all issued first), the rest with one counter atomic.
template <int N>
__device__ __forceinline__ void queue_push_many(const Args& a, const bool (&want)[N], const int (&u)[N],
                                                const Out& o) {
  int nch[N];
#pragma unroll
  for (int q = 0; q < N; ++q) {
    nch[q] = 0;
    if (want[q]) {
      const int d = a.off[u[q] + 1] - a.off[u[q]];
      if (d > a.hub_deg) nch[q] = (d + a.hub_chunk - 1) / a.hub_chunk;
    }
  }
  bool nr[N];
#pragma unroll
  for (int q = 0; q < N; ++q) {
    if (nch[q]) {
      const unsigned long long old = atomicAdd(o.hnext, (1ull << 32) | (unsigned long long)nch[q]);
      const int idx = (int)(old >> 32);
      put(a, o.HV, idx, u[q]);
      put(a, o.HB, idx, (int)(old & 0xffffffffull));
    }
    nr[q] = want[q] && nch[q] == 0;
  }
  warp_push_many<N>(a, nr, u, o.QN, o.qnext);
}

// Pushes of one group: below-threshold improvements to the ring (LOCAL) or the next
// round's queue, far ones to the far pile.
template <bool LOCAL, int N>
__device__ __forceinline__ void push_group(const Args& a, const int (&res)[N], const int (&u)[N], int round,
                                           const Out& o, Ring& r) {
  bool nr[N], fr[N];
#pragma unroll
  for (int q = 0; q < N; ++q) {
    nr[q] = res[q] == 1;
    fr[q] = res[q] == 2;
  }
  if (LOCAL) {
#pragma unroll
    for (int q = 0; q < N; ++q) push_near<true>(a, nr[q], u[q], round, o, r);
  } else {
    queue_push_many<N>(a, nr, u, o);
  }
  warp_push_many<N>(a, fr, u, o.F, o.fcnt);
}

// Relax the out-edges of the warp's batch: lane i holds frontier vertex v (or -1).
// Lane i's edges take positions [excl_i, excl_i + d_i) of the flattened batch; in a
// step, lane t relaxes position t0 + t, owned by the last lane j with excl_j <= t0 + t
// (a lane of degree 0 is never that last lane). LOCAL also sends vertices above
// hub_deg (which only the ring can hold) to the next round's hub list. `work` counts
// the edges relaxed.
template <bool LOCAL>
__device__ __forceinline__ void relax_batch(const Args& a, int v, long long thr, int round, int epoch, const Out& o,
                                            Ring& r, int& work) {
  const int lane = threadIdx.x & 31;
  int b = 0, d = 0;
  long long dv = 0;
  bool hub = false;
  if (v >= 0) {
    // dist[v] is loaded with the offsets, not after the hub test; it is first needed
    // after the adjacency loads below are issued
    b = a.off[v];
    const int e = a.off[v + 1];
    dv = __ldcg(a.dist + v);
    d = e - b;
    if (LOCAL && d > a.hub_deg) {
      hub = true;
      d = 0;
    }
  }
  if (LOCAL) queue_push(a, hub && mark(qbits(a, round + 1), v), v, o.QN, o.qnext, o.HV, o.HB, o.hnext);
  int inc = d;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const int t = __shfl_up_sync(FULL, inc, k);
    if (lane >= k) inc += t;
  }
  const int total = __shfl_sync(FULL, inc, 31);
  const int excl = inc - d;
  work += total;
  for (int t0 = 0; t0 < total; t0 += 32 * SU) {
    int u[SU], res[SU], wt[SU], jq[SU];
    long long nd[SU];
#pragma unroll
    for (int q = 0; q < SU; ++q) {
      const int t = t0 + 32 * q + lane;
      int j = 0;
#pragma unroll
      for (int k = 16; k > 0; k >>= 1)
        if (__shfl_sync(FULL, excl, j + k) <= t) j += k;
      const int jb = __shfl_sync(FULL, b, j);
      const int je = __shfl_sync(FULL, excl, j);
      jq[q] = j;
      u[q] = 0;
      wt[q] = 0;
      if (t < total) {
        const int k = jb + (t - je);
        u[q] = ld_stream(a.adj + k);
        wt[q] = ld_stream(a.w + k);
      }
    }
#pragma unroll
    for (int q = 0; q < SU; ++q) {
      const long long jd = __shfl_sync(FULL, dv, jq[q]);
      nd[q] = t0 + 32 * q + lane < total ? jd + wt[q] : (long long)INT_MAX;
    }
    relax_group<!LOCAL, SU>(a, u, nd, thr, round, epoch, o.fmin, res);
    push_group<LOCAL, SU>(a, res, u, round, o, r);
  }
}

// Edges [vb, ve) of one vertex at distance vd, 32 per step (a hub piece).
template <bool LOCAL>
__device__ __forceinline__ void relax_range(const Args& a, int vb, int ve, long long vd, long long thr, int round,
                                            int epoch, const Out& o, Ring& r) {
  const int lane = threadIdx.x & 31;
  for (int k0 = vb; k0 < ve; k0 += 32 * SU) {
    int u[SU], res[SU];
    long long nd[SU];
#pragma unroll
    for (int q = 0; q < SU; ++q) {
      const int k = k0 + 32 * q + lane;
      u[q] = 0;
      nd[q] = INT_MAX;
      if (k < ve) {
        u[q] = ld_stream(a.adj + k);
        nd[q] = vd + ld_stream(a.w + k);
      }
    }
    relax_group<!LOCAL, SU>(a, u, nd, thr, round, epoch, o.fmin, res);
    push_group<LOCAL, SU>(a, res, u, round, o, r);
  }
}

// Warp-local cascade: relax the ring, 32 entries at a time, until it is empty or the
// warp has relaxed a.local_edges edges; what is left goes to the next round's queue.
// Each pass either relaxes edges (work grows) or only pops, so the loop ends.
__device__ __forceinline__ void cascade(const Args& a, long long thr, int round, int epoch, const Out& o, Ring& r,
                                        int& relaxed) {
  const int lane = threadIdx.x & 31;
  int work = 0;
  while (r.cnt > 0 && work < a.local_edges) {
    __syncwarp();
    const int take = min(r.cnt, 32);
    const int v = lane < take ? r.s[(r.head + lane) & (RING - 1)] : -1;
    __syncwarp();
    r.head = (r.head + take) & (RING - 1);
    r.cnt -= take;
    relax_batch<true>(a, v, thr, round, epoch, o, r, work);
  }
  relaxed += work;
  __syncwarp();
  for (int i0 = 0; i0 < r.cnt; i0 += 32) {
    const int i = i0 + lane;
    int u = 0;
    bool want = false;
    if (i < r.cnt) {
      u = r.s[(r.head + i) & (RING - 1)];
      want = mark(qbits(a, round + 1), u);
    }
    queue_push(a, want, u, o.QN, o.qnext, o.HV, o.HB, o.hnext);
  }
  __syncwarp();
  r.head = 0;
  r.cnt = 0;
}

// The inputs of the per-epoch width choice for candidate factor f (all from values
// every CTA of the solve reads identically after a barrier).
__device__ __forceinline__ void epoch_inputs(const Args& a, int f, float fn, float rounds_prev, float relaxed_prev,
                                             int epoch, int f_prev, float progress, float* x) {
  x[0] = a.sfeat[0];
  x[1] = a.sfeat[1];
  x[2] = a.sfeat[2];
  x[3] = a.sfeat[3];
  x[4] = log2f(1.0f + fn);            // far pile at this advance
  x[5] = x[4] - a.sfeat[0];           // ... as a fraction of V (log)
  x[6] = log2f(1.0f + rounds_prev);   // relax rounds of the previous epoch
  x[7] = log2f(1.0f + relaxed_prev);  // edges relaxed in the previous epoch
  x[8] = log2f(1.0f + (float)epoch);
  x[9] = log2f((float)kFacNum[f_prev]) - 2.0f;  // previous width factor (log2)
  x[10] = log2f((float)kFacNum[f]) - 2.0f;      // candidate width factor (log2)
  x[11] = x[10] * x[4];
  x[12] = progress;                   // log2(1 + smallest far distance / largest weight)
}

// The width factor the epoch model scores lowest (predicted log cost per unit of
// distance): NFAC candidates x 32 hidden units over the CTA's threads, every CTA
// evaluating the same inputs with the same instructions in the same order, so all
// pick the same factor without a barrier between them. Ties go to the smaller factor.
__device__ int epoch_choice(const Args& a, float fn, float rounds_prev, float relaxed_prev, int epoch, int f_prev,
                            float progress) {
  __shared__ float s_x[NFAC][SP_MLP_IN];
  if (threadIdx.x < NFAC)
    epoch_inputs(a, threadIdx.x, fn, rounds_prev, relaxed_prev, epoch, f_prev, progress, s_x[threadIdx.x]);
  return mlp_argmin<NFAC>(a.emodel, s_x, a.ewiden ? 2 : 0);
}

// One delta-stepping solve by `nblk` co-resident CTAs (this one is number `blk`):
// the whole grid for a single source, or one group of a batched launch.
__device__ __forceinline__ void delta_run(const Args& a, const int blk, const int nblk, int32_t* ring) {
  Ctl* c = a.ctl;
  const int lane = threadIdx.x & 31;
  const int gw = (blk * THREADS + threadIdx.x) >> 5;
  const int nw = (nblk * THREADS) >> 5;
  int round = 0, epoch = 0;
  long long thr = a.delta;  // bucket 0 = [0, delta)
  // per-epoch width state (identical in every CTA of the solve)
  int f_prev = 2, round_mark = 0;
  unsigned long long relaxed_mark = 0;
  while (true) {
    // counts clamped to the buffers (an overflow was already flagged by put())
    const int qv = min(*(volatile int*)&c->qcount[round % 3], a.V);
    const unsigned long long hc = *(volatile unsigned long long*)&c->hcount[round % 3];
    const int hn = min((int)(hc >> 32), a.V), hchunks = (int)(hc & 0xffffffffull);
    const int qn = qv;
    const int fn = min(*(volatile int*)&c->fcount[epoch % 3], a.V);
    if (qv == 0 && hn == 0 && fn == 0) break;
    if ((long long)round >= a.max_rounds) {
      if (blk == 0 && threadIdx.x == 0) c->status = 1;
      break;
    }
    // this phase marks round + 1 (and the current epoch); the marks of `round` are
    // tested by no one from here on: clear them for round + 2
    for (int i = blk * THREADS + threadIdx.x; i < a.nwords; i += nblk * THREADS) qbits(a, round)[i] = 0u;
    if (qv > 0 || hn > 0) {
      const int32_t* Q = a.q[round & 1];
      const Out o = {a.q[(round + 1) & 1], &c->qcount[(round + 1) % 3], a.hv[(round + 1) & 1],
                     a.hbase[(round + 1) & 1], &c->hcount[(round + 1) % 3], a.f[epoch & 1], &c->fcount[epoch % 3],
                     &c->fmin[epoch % 3]};
      Ring r = {ring + (threadIdx.x >> 5) * RING, 0, 0};
      // a small frontier is spread over all warps (fewer entries per warp, fewer steps)
      const int per = min(32, max(1, (qn + nw - 1) / nw));
      const bool local = a.local_edges > 0 && qn <= nw * 32;
      int work = 0;
      for (int base = gw * per; base < qn; base += nw * per) {
        const int v = (lane < per && base + lane < qn) ? Q[base + lane] : -1;
        if (local)
          relax_batch<true>(a, v, thr, round, epoch, o, r, work);
        else
          relax_batch<false>(a, v, thr, round, epoch, o, r, work);
      }
      // hub pieces of this round: hub_chunk edges per warp, all warps
      {
        const int32_t* HVc = a.hv[round & 1];
        const int32_t* HBc = a.hbase[round & 1];
        for (int ch = gw; ch < hchunks; ch += nw) {
          int lo = 0, hi = hn - 1;  // last entry whose first chunk <= ch
          while (lo < hi) {
            const int m = (lo + hi + 1) >> 1;
            if (HBc[m] <= ch) lo = m; else hi = m - 1;
          }
          const int v = HVc[lo];
          const long long vd = __ldcg(a.dist + v);
          const int vb = a.off[v] + (ch - HBc[lo]) * a.hub_chunk;
          const int ve = min(vb + a.hub_chunk, a.off[v + 1]);
          work += max(0, ve - vb);
          if (local)
            relax_range<true>(a, vb, ve, vd, thr, round, epoch, o, r);
          else
            relax_range<false>(a, vb, ve, vd, thr, round, epoch, o, r);
        }
      }
      if (local) cascade(a, thr, round, epoch, o, r, work);
      if (lane == 0 && work > 0) atomicAdd(&c->relaxed, (unsigned long long)work);
      if (blk == 0 && threadIdx.x == 0) {
        c->qcount[(round + 2) % 3] = 0;  // read two rounds ago
        c->hcount[(round + 2) % 3] = 0ull;
      }
      if (!group_barrier(&c->bar, (unsigned)nblk, blk == 0)) break;
      ++round;
    } else {
      // bucket advance: threshold to the bucket after the smallest far distance
      const long long fm = *(volatile int*)&c->fmin[epoch % 3];
      const long long thr_old = thr;
      long long w = a.delta;
      if (a.epolicy != 0 && a.delta < (long long)INT_MAX) {
        const unsigned long long rel = *(volatile unsigned long long*)&c->relaxed;
        const float rounds_prev = (float)(round - round_mark), relaxed_prev = (float)(rel - relaxed_mark);
        const float progress = log2f(1.0f + (float)fm / fmaxf(1.0f, exp2f(a.sfeat[3])));
        int f;
        if (a.epolicy == 2) {
          unsigned h = a.eseed * 0x9e3779b9u ^ ((unsigned)epoch * 0x85ebca6bu);
          h ^= h >> 15;
          h *= 0x2c1b3c6du;
          h ^= h >> 12;
          f = (int)(h % NFAC);
        } else {
          f = epoch_choice(a, (float)fn, rounds_prev, relaxed_prev, epoch, f_prev, progress);
        }
        w = max(1ll, a.delta * kFacNum[f] / 4);
        if (a.etrace && blk == 0 && threadIdx.x == 0 && epoch < a.etrace_cap) {
          float x[SP_MLP_IN];
          epoch_inputs(a, f, (float)fn, rounds_prev, relaxed_prev, epoch, f_prev, progress, x);
          float* r = a.etrace + (size_t)epoch * ETRACE;
          for (int i = 0; i < SP_MLP_IN; ++i) r[i] = x[i];
          r[SP_MLP_IN] = (float)kFacNum[f] / 4.0f;
          const long long t_new = max((fm / w + 1) * w, thr_old + w);
          r[SP_MLP_IN + 1] = (float)(t_new - thr_old);
          unsigned long long now;
          asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
          a.etime[epoch] = now;
        }
        f_prev = f;
        round_mark = round;
        relaxed_mark = rel;
      }
      thr = (a.delta >= (long long)INT_MAX) ? (long long)INT_MAX + 1 : (fm / w + 1) * w;
      if (thr <= thr_old) thr = thr_old + w;
      // The split fills the queue of the NEXT round (its own counter slot): every
      // phase decision reads qcount[round % 3], and no phase may write the slot its
      // own decision read while slower CTAs may still be reading it.
      // the split marks epoch + 1; nothing tests this epoch's far marks any more
      for (int i = blk * THREADS + threadIdx.x; i < a.nwords; i += nblk * THREADS) fbits(a, epoch)[i] = 0u;
      const int32_t* F = a.f[epoch & 1];
      int32_t* FN = a.f[(epoch + 1) & 1];
      int* fnext = &c->fcount[(epoch + 1) % 3];
      int* fminn = &c->fmin[(epoch + 1) % 3];
      int32_t* Q = a.q[(round + 1) & 1];
      int* qcnt = &c->qcount[(round + 1) % 3];
      int32_t* HV = a.hv[(round + 1) & 1];
      int32_t* HB = a.hbase[(round + 1) & 1];
      unsigned long long* hnext = &c->hcount[(round + 1) % 3];
      for (int base = gw * 32; base < fn; base += nw * 32) {
        const int i = base + lane;
        bool toq = false, tof = false;
        int u = 0;
        if (i < fn) {
          u = F[i];
          const int du = __ldcg(a.dist + u);
          if ((long long)du >= thr_old) {  // below thr_old: already settled through the queue
            if ((long long)du < thr) {
              toq = mark(qbits(a, round + 1), u);
            } else {
              tof = mark(fbits(a, epoch + 1), u);
              if (tof) atomicMin(fminn, du);
            }
          }
        }
        queue_push(a, toq, u, Q, qcnt, HV, HB, hnext);
        warp_push(a, tof, u, FN, fnext);
      }
      if (blk == 0 && threadIdx.x == 0) {
        c->fcount[(epoch + 2) % 3] = 0;
        c->fmin[(epoch + 2) % 3] = INT_MAX;
        c->qcount[(round + 2) % 3] = 0;  // read two phases ago
        c->hcount[(round + 2) % 3] = 0ull;
      }
      if (!group_barrier(&c->bar, (unsigned)nblk, blk == 0)) break;
      ++epoch;
      ++round;
    }
  }
  if (blk == 0 && threadIdx.x == 0) {
    c->rounds = round - epoch;  // relax rounds (each split also consumed a round number)
    if (a.etrace && epoch <= a.etrace_cap) {  // the end of the last traced epoch
      unsigned long long now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      a.etime[min(epoch, a.etrace_cap)] = now;
    }
    c->epochs = epoch;
    if (c->bar.error) c->status = 1;
  }
}

__global__ void __launch_bounds__(THREADS, 4) k_delta(Args a) {
  __shared__ int32_t ring[(THREADS / 32) * RING];
  delta_run(a, blockIdx.x, gridDim.x, ring);
}

// Many sources in one cooperative launch: CTA group g = blockIdx.x / gsz solves the
// g-th source of the batch over its own V-strided slice of every per-vertex buffer
// and its own Ctl (counters, bounded group barrier). Adjacency, weights and offsets
// are shared, so the groups' gathers share L2.
__global__ void __launch_bounds__(THREADS, 4) k_delta_multi(Args a, int gsz) {
  __shared__ int32_t ring[(THREADS / 32) * RING];
  __shared__ Args b;  // this group's arguments (shared: read like the kernel parameters)
  const int g = blockIdx.x / gsz;
  if (threadIdx.x == 0) {
    const size_t o = (size_t)g * (size_t)a.V;
    b = a;
    b.dist += o;
    for (int k = 0; k < 2; ++k) {
      b.q[k] += o;
      b.f[k] += o;
      b.hv[k] += o;
      b.hbase[k] += o;
    }
    b.bits += (size_t)g * 4 * a.nwords;
    b.ctl += g;
  }
  __syncthreads();
  delta_run(b, blockIdx.x % gsz, gsz, ring);
}

// Initial state of a solve from src (the mark bitmaps are zeroed by the host).
__global__ void k_init(int V, int src, int32_t* dist, int32_t* q0, int32_t* hv0, int32_t* hb0,
                       const int32_t* __restrict__ off, Ctl* c, int hub_deg, int hub_chunk) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) dist[v] = v == src ? 0 : INT_MAX;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->bar.arrived = 0;
    c->bar.error = 0;
    for (int k = 0; k < 3; ++k) {
      c->qcount[k] = 0;
      c->hcount[k] = 0ull;
    }
    const int d = off[src + 1] - off[src];
    if (d > hub_deg) {
      hv0[0] = src;
      hb0[0] = 0;
      c->hcount[0] = (1ull << 32) | (unsigned long long)((d + hub_chunk - 1) / hub_chunk);
    } else {
      q0[0] = src;
      c->qcount[0] = 1;
    }
    for (int k = 0; k < 3; ++k) {
      c->fcount[k] = 0;
      c->fmin[k] = INT_MAX;
    }
    c->rounds = c->epochs = c->status = 0;
    c->relaxed = 0ull;
  }
}

// Initial state of every source of a batch: blockIdx.y = position in the batch, each
// with its V-strided slices and its own Ctl (as k_init for one source).
__global__ void k_init_multi(int V, const int32_t* __restrict__ srcs, int32_t* dist, int32_t* q0, int32_t* hv0,
                             int32_t* hb0, const int32_t* __restrict__ off, Ctl* ctl, int hub_deg, int hub_chunk) {
  const int g = blockIdx.y;
  const size_t o = (size_t)g * (size_t)V;
  const int src = srcs[g];
  dist += o;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) dist[v] = v == src ? 0 : INT_MAX;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    Ctl* c = ctl + g;
    c->bar.arrived = 0;
    c->bar.error = 0;
    for (int k = 0; k < 3; ++k) {
      c->qcount[k] = 0;
      c->hcount[k] = 0ull;
      c->fcount[k] = 0;
      c->fmin[k] = INT_MAX;
    }
    const int d = off[src + 1] - off[src];
    if (d > hub_deg) {
      hv0[o] = src;
      hb0[o] = 0;
      c->hcount[0] = (1ull << 32) | (unsigned long long)((d + hub_chunk - 1) / hub_chunk);
    } else {
      q0[o] = src;
      c->qcount[0] = 1;
    }
    c->rounds = c->epochs = c->status = 0;
    c->relaxed = 0ull;
  }
}

// Warm start (sp_sssp_dynamic): dist keeps the caller's values; the counters are reset
// here (the host zeroes the mark bitmaps), and k_seed then queues the seed vertices
// (hubs as hub entries).
__global__ void k_reset(Ctl* c) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->bar.arrived = 0;
    c->bar.error = 0;
    for (int k = 0; k < 3; ++k) {
      c->qcount[k] = 0;
      c->hcount[k] = 0ull;
      c->fcount[k] = 0;
      c->fmin[k] = INT_MAX;
    }
    c->rounds = c->epochs = c->status = 0;
    c->relaxed = 0ull;
  }
}

// Queues n distinct seeds for round 0 (after k_reset, in stream order).
__global__ void k_seed(int n, const int32_t* __restrict__ seeds, int32_t* q0, int32_t* hv0,
                       int32_t* hb0, const int32_t* __restrict__ off, Ctl* c, int hub_deg, int hub_chunk) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = seeds[i];
    const int d = off[v + 1] - off[v];
    if (d > hub_deg) {
      const unsigned long long old =
          atomicAdd(&c->hcount[0], (1ull << 32) | (unsigned long long)((d + hub_chunk - 1) / hub_chunk));
      hv0[old >> 32] = v;
      hb0[old >> 32] = (int)(old & 0xffffffffull);
    } else {
      q0[atomicAdd(&c->qcount[0], 1)] = v;
    }
  }
}

// ---- plain form (generated CUDA code shape)
__global__ void k_plain(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                        const int32_t* __restrict__ w, int32_t* dist, const char* __restrict__ modified,
                        char* __restrict__ modified_nxt, int* finished) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V || !modified[v]) return;
  for (int e = off[v]; e < off[v + 1]; ++e) {
    int nbr = adj[e];
    long long nd = (long long)dist[v] + w[e];
    if (nd < INT_MAX && dist[nbr] > (int)nd) {
      int old = atomicMin(&dist[nbr], (int)nd);
      if (old > (int)nd) {
        modified_nxt[nbr] = 1;
        *finished = 0;
      }
    }
  }
}

__global__ void k_plain_init(int V, int src, int32_t* dist, char* m, char* mn) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < V) {
    dist[v] = v == src ? 0 : INT_MAX;
    m[v] = v == src;
    mn[v] = 0;
  }
}

__global__ void k_minmax_w(const int32_t* __restrict__ w, int64_t E, int* mn, int* mx) {
  int lo = INT_MAX, hi = INT_MIN;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    lo = min(lo, w[e]);
    hi = max(hi, w[e]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mn, lo);
    atomicMax(mx, hi);
  }
}

// ---- decremental repair of a batch with deletions (positive weights)
__global__ void k_fill(int n, int32_t* a, int32_t val) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = val;
}

// parent[v] = the smallest u with d[u] + w(u, v) == d[v] (a tight in-edge), INT_MAX for
// none (the source, unreachable vertices). With every weight >= 1, tight edges raise the
// distance, so the parents form a forest.
__global__ void k_parents(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                          const int32_t* __restrict__ w, const int32_t* __restrict__ d, int32_t* parent) {
  const int lane = threadIdx.x & 31;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < V; u += (gridDim.x * blockDim.x) >> 5) {
    const int du = d[u];
    if (du == INT_MAX) continue;
    for (int j = off[u] + lane; j < off[u + 1]; j += 32) {
      const int v = adj[j];
      if ((long long)du + w[j] == (long long)d[v]) atomicMin(parent + v, u);
    }
  }
}

// A record (s, t) of the batch on t's parent edge (deleted, or lengthened by an added
// weight) leaves t's distance unsupported: t is marked.
__global__ void k_mark_parent_edges(int n, const int32_t* __restrict__ s, const int32_t* __restrict__ t,
                                    const int32_t* __restrict__ parent, int V, uint8_t* bad, int* nbad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ti = t[i];
    if (ti >= 0 && ti < V && parent[ti] == s[i] && bad[ti] == 0) {
      bad[ti] = 1;
      atomicAdd(nbad, 1);
    }
  }
}

// Ancestor links for pointer jumping: the parent, or the vertex itself at a root.
__global__ void k_anc_init(int V, const int32_t* __restrict__ parent, int32_t* anc) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    anc[v] = parent[v] == INT_MAX ? v : parent[v];
}

// One synchronous pointer-jumping pass (inputs and outputs in separate buffers): after
// pass k, bad[v] covers v's 2^k nearest ancestors and anc[v] is its 2^k-th ancestor (or
// its root), so ceil(log2 V) + 1 passes cover every chain. An in-place pass is not
// enough: a link can jump past an ancestor whose mark is set later in the same pass.
__global__ void k_jump(int V, const int32_t* __restrict__ anc_in, const uint8_t* __restrict__ bad_in,
                       int32_t* __restrict__ anc_out, uint8_t* __restrict__ bad_out) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int a = anc_in[v];
    bad_out[v] = bad_in[v] | bad_in[a];
    anc_out[v] = anc_in[a];
  }
}

__global__ void k_reset_marked(int V, const uint8_t* __restrict__ bad, int32_t* dist) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    if (bad[v]) dist[v] = INT_MAX;
}

// Edges of the updated graph from unmarked vertices into marked ones lower the marked
// ends (the unmarked distances are still achievable and are not changed here).
__global__ void k_push_into_marked(int V, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                   const int32_t* __restrict__ w, const uint8_t* __restrict__ bad, int32_t* dist) {
  const int lane = threadIdx.x & 31;
  for (int y = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; y < V; y += (gridDim.x * blockDim.x) >> 5) {
    if (bad[y]) continue;
    const int dy = dist[y];
    if (dy == INT_MAX) continue;
    for (int j = off[y] + lane; j < off[y + 1]; j += 32) {
      const int x = adj[j];
      if (!bad[x]) continue;
      const long long nd = (long long)dy + w[j];
      if (nd < (long long)INT_MAX) atomicMin(dist + x, (int)nd);
    }
  }
}

// The marked vertices that now have a finite distance: the repair's seeds.
__global__ void k_collect_marked(int V, const uint8_t* __restrict__ bad, const int32_t* __restrict__ dist,
                                 int32_t* seeds, int* nseeds) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    if (bad[v] && dist[v] != INT_MAX) seeds[atomicAdd(nseeds, 1)] = v;
}

__global__ void k_count_marked(int V, const uint8_t* __restrict__ bad, int* count) {
  int c = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) c += bad[v];
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

}  // namespace ss

struct SsspPlan {
  dbuf<int32_t> dist, q0, q1, f0, f1, wbuf, h0, h1, hb0, hb1;
  dbuf<unsigned> bits;  // the four mark bitmaps
  dbuf<char> m0, m1;
  dbuf<ss::Ctl> ctl;
  dbuf<int> tmp;
  const void* w_src = nullptr;  // weights cached in wbuf came from this pointer
  int w_min = 0, w_max = 0;
  // the learned choice of the last call: its inputs are the graph and the weight range
  // only, so it is reused while the range and the loaded model stay the same
  unsigned sel_gen = 0;
  int sel_wmin = 0, sel_wmax = 0, sel_ctas = 0, sel_local = 0, sel_local_knob = -1;
  int64_t sel_delta = 0;
  // the per-epoch width model on the device (uploaded when its generation changes) and
  // the trace of the last traced solve
  dbuf<float> emodel;
  unsigned emodel_gen = 0;
  dbuf<float> etrace;
  dbuf<unsigned long long> etime;
  int etrace_n = 0;
};

void free_sssp_plan(SsspPlan* p) { delete p; }

unsigned mlp_epoch_model(std::vector<float>& packed);  // sp_mlp.cu
constexpr int ETRACE_CAP = 1 << 16;                     // traced epochs per solve

// The per-epoch width fields of a: the policy (knob sssp.epoch; by default learned when
// an epoch model is loaded), the model on the device, the static inputs, and the trace
// buffers when tracing a single-source solve.
static int epoch_setup(sp_graph* g, ss::Args& a, bool trace) {
  SsspPlan* p = g->sssp;
  std::vector<float> packed;
  const unsigned gen = mlp_epoch_model(packed);
  int pol = g->sssp_epoch;
  if (pol < 0) pol = gen ? 1 : 0;
  if (pol == 1 && !gen) pol = 0;  // no model: the fixed width
  a.epolicy = pol;
  a.ewiden = g->sssp_epoch_widen;
  a.eseed = (unsigned)g->sssp_epoch_seed;
  a.emodel = nullptr;
  a.etrace = nullptr;
  a.etime = nullptr;
  a.etrace_cap = 0;
  if (pol == 1) {
    if (p->emodel_gen != gen) {
      SP_TRY(p->emodel.alloc(packed.size()));
      SP_CHECK_CUDA(cudaMemcpyAsync(p->emodel.p, packed.data(), sizeof(float) * packed.size(),
                                    cudaMemcpyHostToDevice, g->stream));
      p->emodel_gen = gen;
    }
    a.emodel = p->emodel.p;
  }
  const double V = std::max(1, g->V), E = (double)g->E;
  a.sfeat[0] = (float)std::log2(V);
  a.sfeat[1] = (float)std::log2(E + 1.0);
  a.sfeat[2] = (float)(E / V);
  a.sfeat[3] = (float)std::log2(std::max(1.0, (double)p->w_max));
  if (trace && pol != 0) {
    SP_TRY(p->etrace.alloc((size_t)ETRACE_CAP * ss::ETRACE));
    SP_TRY(p->etime.alloc((size_t)ETRACE_CAP + 1));
    a.etrace = p->etrace.p;
    a.etime = p->etime.p;
    a.etrace_cap = ETRACE_CAP;
  }
  g->sssp_last_epolicy = pol;
  return SP_OK;
}
int sssp_hub_deg_default() { return ss::HUB_DEG; }
int sssp_hub_chunk_default() { return ss::HUB_CHUNK; }
int sssp_local_default() { return ss::LOCAL_STEPS; }

static int sssp_prepare(sp_graph* g, const int32_t* weight, const int32_t** wdev) {
  if (!g->sssp) g->sssp = new SsspPlan();
  SsspPlan* p = g->sssp;
  cudaStream_t s = g->stream;
  const int32_t* w = nullptr;
  if (weight) {
    SP_TRY(p->wbuf.alloc(g->E));
    if (g->E) SP_CHECK_CUDA(cudaMemcpyAsync(p->wbuf.p, weight, sizeof(int32_t) * g->E, cudaMemcpyDefault, s));
    w = p->wbuf.p;
  } else if (g->has_w) {
    w = g->w.p;
  } else {
    set_error("sp_sssp: no weights given and the graph has no edgeLen");
    return SP_ERR_INVALID;
  }
  SP_TRY(p->tmp.alloc(2));
  int init[2] = {INT_MAX, INT_MIN};
  SP_CHECK_CUDA(cudaMemcpyAsync(p->tmp.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
  if (g->E) {
    ss::k_minmax_w<<<num_sms() * 4, 256, 0, s>>>(w, g->E, p->tmp.p, p->tmp.p + 1);
    SP_CHECK_LAUNCH();
  }
  int mm[2];
  SP_TRY(copy_out(mm, p->tmp.p, sizeof(mm), s));
  p->w_min = g->E ? mm[0] : 0;
  p->w_max = g->E ? mm[1] : 0;
  *wdev = w;
  return SP_OK;
}

int mlp_score(const std::vector<float>& X, std::vector<float>& y, cudaStream_t s);
unsigned mlp_generation();  // 0 = no model loaded

// Scheduler inputs (SP_MLP_IN): graph shape and weight range, then the candidate
// schedule (log2 of the delta multiple of the largest weight, CTAs per SM, warp
// cascade budget).
static int sssp_features(sp_graph* g, double mult, int ctas, int local, float* x) {
  SP_TRY(ensure_symmetry(g));
  const double V = g->V, E = (double)g->E, avg = E / V;
  const double mx = g->max_out_deg, wmax = std::max(1, g->sssp->w_max), wmin = g->sssp->w_min;
  x[0] = (float)std::log2(V);
  x[1] = (float)std::log2(E + 1.0);
  x[2] = (float)avg;
  x[3] = (float)std::log2(mx + 1.0);
  x[4] = (float)std::log2((mx + 1.0) / (avg + 1.0));
  x[5] = (float)g->symmetric;
  x[6] = (float)std::log2(wmax + 1.0);
  x[7] = (float)std::log2(std::max(1.0, wmax - wmin + 1.0));
  x[8] = (float)std::log2(mult);
  x[9] = (float)ctas;
  x[10] = (float)(std::log2(mult) * std::log2(V));  // interaction: bucket width vs size
  x[11] = (float)(ctas * avg);
  x[12] = (float)std::log2(1.0 + local);
  return SP_OK;
}

// One delta-stepping solve from src, or (warm, nseeds > 0) from the distances already
// in the plan's dist buffer with the given device seed vertices queued.
static int sssp_delta(sp_graph* g, const int32_t* w, int32_t src, int32_t* dist_out, int64_t delta, int ctas,
                      int local, int32_t* rounds_out, const int32_t* d_seeds = nullptr, int nseeds = 0) {
  SsspPlan* p = g->sssp;
  cudaStream_t s = g->stream;
  const int V = g->V;
  SP_TRY(p->dist.alloc(V));
  SP_TRY(p->q0.alloc(V));
  SP_TRY(p->q1.alloc(V));
  SP_TRY(p->f0.alloc(V));
  SP_TRY(p->f1.alloc(V));
  const int nwords = (V + 31) / 32;
  SP_TRY(p->bits.alloc((size_t)4 * nwords));
  SP_CHECK_CUDA(cudaMemsetAsync(p->bits.p, 0, sizeof(unsigned) * 4 * (size_t)nwords, s));
  SP_TRY(p->h0.alloc(V));
  SP_TRY(p->h1.alloc(V));
  SP_TRY(p->hb0.alloc(V));
  SP_TRY(p->hb1.alloc(V));
  SP_TRY(p->ctl.alloc(1));
  const bool negative = p->w_min < 0;
  if (negative || delta <= 0) delta = negative ? (int64_t)INT_MAX : std::max<int64_t>(1, delta);
  ss::Args a;
  a.off = g->off.p;
  a.adj = g->adj.p;
  a.w = w;
  a.dist = p->dist.p;
  a.q[0] = p->q0.p;
  a.q[1] = p->q1.p;
  a.f[0] = p->f0.p;
  a.f[1] = p->f1.p;
  a.hv[0] = p->h0.p;
  a.hv[1] = p->h1.p;
  a.hbase[0] = p->hb0.p;
  a.hbase[1] = p->hb1.p;
  a.bits = p->bits.p;
  a.nwords = nwords;
  a.ctl = p->ctl.p;
  a.V = V;
  a.delta = delta;
  // Bellman-Ford needs at most V-1 rounds of improvement per vertex chain; far more
  // rounds than V * 4 + 64 can only come from a negative cycle.
  a.max_rounds = (long long)V * 4 + 64;
  a.hub_deg = std::min(g->sssp_hub_deg > 0 ? g->sssp_hub_deg : ss::HUB_DEG, ss::HUB_DEG_MAX);
  a.hub_chunk = g->sssp_hub_chunk > 0 ? g->sssp_hub_chunk : ss::HUB_CHUNK;
  a.local_edges = 32 * local;
  a.filter = g->sssp_filter;
  SP_TRY(epoch_setup(g, a, g->sssp_trace != 0));
  if (nseeds > 0) {
    ss::k_reset<<<1, 32, 0, s>>>(p->ctl.p);
    SP_CHECK_LAUNCH();
    ss::k_seed<<<std::max(1, std::min(num_sms() * 4, (nseeds + 255) / 256)), 256, 0, s>>>(
        nseeds, d_seeds, p->q0.p, p->h0.p, p->hb0.p, g->off.p, p->ctl.p, a.hub_deg, a.hub_chunk);
    SP_CHECK_LAUNCH();
  } else {
    ss::k_init<<<num_sms() * 4, 256, 0, s>>>(V, src, p->dist.p, p->q0.p, p->h0.p, p->hb0.p, g->off.p, p->ctl.p,
                                              a.hub_deg, a.hub_chunk);
    SP_CHECK_LAUNCH();
  }
  int per_sm = 0;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ss::k_delta, ss::THREADS, 0));
  const int grid = num_sms() * std::max(1, std::min(per_sm, ctas));
  void* params[] = {&a};
  SP_CHECK_CUDA(cudaLaunchCooperativeKernel((void*)ss::k_delta, grid, ss::THREADS, params, 0, s));
  g_launches++;
  ss::Ctl hc;
  SP_TRY(copy_out(&hc, p->ctl.p, sizeof(hc), s));
  if (rounds_out) *rounds_out = hc.rounds;
  if (nseeds == 0) g->sssp_last_rounds = hc.rounds;  // a solve from the source
  g->sssp_last_relaxed = (int64_t)hc.relaxed;
  g->sssp_last_epochs = hc.epochs;
  p->etrace_n = a.etrace ? std::min(hc.epochs, ETRACE_CAP) : 0;
  if (hc.status == 3) {
    set_error("sp_sssp: a queue overflowed its V entries (internal error; distances not valid)");
    return SP_ERR_CUDA;
  }
  if (hc.status != 0 || hc.bar.error) {
    if (negative && !hc.bar.error) {
      set_error("sp_sssp: no fixed point after %d rounds (negative cycle)", hc.rounds);
      return SP_ERR_NEG_CYCLE;
    }
    set_error("sp_sssp: device loop gave up (status %d, barrier error %d)", hc.status, hc.bar.error);
    return SP_ERR_TIMEOUT;
  }
  if (dist_out) SP_TRY(copy_out(dist_out, p->dist.p, sizeof(int32_t) * V, s));
  return SP_OK;
}

// Many sources, one cooperative launch per batch (k_delta_multi): a batch of B sources
// gives each source a group of gsz = (co-resident CTAs) / B CTAs with its own
// V-strided buffers and Ctl. After each batch, done(rows, b, first) receives the
// device distance rows of its b sources (source-major, V each; `first` = the batch's
// first position in srcs).
int sssp_batch_default() { return ss::BATCH; }

template <class F>
static int sssp_delta_batches(sp_graph* g, const int32_t* w, const std::vector<int32_t>& srcs, int64_t delta,
                              int ctas, int local, F done) {
  SsspPlan* p = g->sssp;
  cudaStream_t s = g->stream;
  const int V = g->V, n = (int)srcs.size();
  if (n == 0) return SP_OK;
  const bool negative = p->w_min < 0;
  if (negative || delta <= 0) delta = negative ? (int64_t)INT_MAX : std::max<int64_t>(1, delta);
  int per_sm = 0;
  SP_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ss::k_delta_multi, ss::THREADS, 0));
  const int total = num_sms() * std::max(1, std::min(per_sm, ctas));
  int B = g->sssp_batch > 0 ? g->sssp_batch : ss::BATCH;
  B = std::max(1, std::min({B, n, total}));
  {  // 9 V-sized int32 buffers and 4 bitmaps per source in flight: keep a batch within
     // 1/8 of device memory
    size_t free_b = 0, total_b = 0;
    SP_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_src = (size_t)9 * 4 * (size_t)V + (size_t)V / 2 + 4096;
    B = (int)std::max<size_t>(1, std::min<size_t>(B, (total_b / 8) / per_src));
  }
  const int gsz = total / B;
  const size_t BV = (size_t)B * V;
  Arena A;
  const int nwords = (V + 31) / 32;
  dspan<int32_t> dist, q0, q1, f0, f1, h0, h1, hb0, hb1, dsrc;
  dspan<unsigned> bits;
  dspan<ss::Ctl> ctl;
  for (dspan<int32_t>* d : {&dist, &q0, &q1, &f0, &f1, &h0, &h1, &hb0, &hb1}) A.want(*d, BV);
  A.want(bits, (size_t)4 * nwords * B);
  A.want(dsrc, B);
  A.want(ctl, B);
  SP_TRY(A.commit());
  ss::Args a;
  a.off = g->off.p;
  a.adj = g->adj.p;
  a.w = w;
  a.dist = dist.p;
  a.q[0] = q0.p;
  a.q[1] = q1.p;
  a.f[0] = f0.p;
  a.f[1] = f1.p;
  a.hv[0] = h0.p;
  a.hv[1] = h1.p;
  a.hbase[0] = hb0.p;
  a.hbase[1] = hb1.p;
  a.bits = bits.p;
  a.nwords = nwords;
  a.ctl = ctl.p;
  a.V = V;
  a.delta = delta;
  a.max_rounds = (long long)V * 4 + 64;
  a.hub_deg = std::min(g->sssp_hub_deg > 0 ? g->sssp_hub_deg : ss::HUB_DEG, ss::HUB_DEG_MAX);
  a.hub_chunk = g->sssp_hub_chunk > 0 ? g->sssp_hub_chunk : ss::HUB_CHUNK;
  a.local_edges = 32 * local;
  a.filter = g->sssp_filter;
  SP_TRY(epoch_setup(g, a, false));
  std::vector<ss::Ctl> hc(B);
  int64_t relaxed = 0;
  for (int k0 = 0; k0 < n; k0 += B) {
    const int b = std::min(B, n - k0);
    SP_CHECK_CUDA(cudaMemcpyAsync(dsrc.p, srcs.data() + k0, sizeof(int32_t) * b, cudaMemcpyHostToDevice, s));
    SP_CHECK_CUDA(cudaMemsetAsync(bits.p, 0, sizeof(unsigned) * 4 * (size_t)nwords * b, s));
    ss::k_init_multi<<<dim3(std::max(1, num_sms() * 4 / b), b), 256, 0, s>>>(
        V, dsrc.p, dist.p, q0.p, h0.p, hb0.p, g->off.p, ctl.p, a.hub_deg, a.hub_chunk);
    SP_CHECK_LAUNCH();
    int gs = gsz;
    void* params[] = {&a, &gs};
    SP_CHECK_CUDA(cudaLaunchCooperativeKernel((void*)ss::k_delta_multi, b * gsz, ss::THREADS, params, 0, s));
    g_launches++;
    SP_TRY(copy_out(hc.data(), ctl.p, sizeof(ss::Ctl) * b, s));
    for (int i = 0; i < b; ++i) {
      relaxed += (int64_t)hc[i].relaxed;
      if (hc[i].status == 3) {
        set_error("sp_sssp_batch: a queue overflowed its V entries for source %d (internal error)", srcs[k0 + i]);
        return SP_ERR_CUDA;
      }
      if (hc[i].status != 0 || hc[i].bar.error) {
        if (negative && !hc[i].bar.error) {
          set_error("sp_sssp: no fixed point from source %d after %d rounds (negative cycle)", srcs[k0 + i],
                    hc[i].rounds);
          return SP_ERR_NEG_CYCLE;
        }
        set_error("sp_sssp: device loop gave up for source %d (status %d, barrier error %d)", srcs[k0 + i],
                  hc[i].status, hc[i].bar.error);
        return SP_ERR_TIMEOUT;
      }
    }
    SP_TRY(done((const int32_t*)dist.p, b, k0));
  }
  g->sssp_last_relaxed = relaxed;
  g->sssp_last_batch = B;
  return SP_OK;
}

static int sssp_plain(sp_graph* g, const int32_t* w, int32_t src, int32_t* dist_out, int32_t* rounds_out) {
  SsspPlan* p = g->sssp;
  cudaStream_t s = g->stream;
  const int V = g->V;
  SP_TRY(p->dist.alloc(V));
  SP_TRY(p->m0.alloc(V));
  SP_TRY(p->m1.alloc(V));
  SP_TRY(p->tmp.alloc(2));
  const int tb = 512, nb = (V + tb - 1) / tb;
  ss::k_plain_init<<<nb, tb, 0, s>>>(V, src, p->dist.p, p->m0.p, p->m1.p);
  SP_CHECK_LAUNCH();
  char* m = p->m0.p;
  char* mn = p->m1.p;
  int rounds = 0;
  const int max_rounds = V + 1;
  while (true) {
    int one = 1;
    SP_CHECK_CUDA(cudaMemcpyAsync(p->tmp.p, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    ss::k_plain<<<nb, tb, 0, s>>>(V, g->off.p, g->adj.p, w, p->dist.p, m, mn, p->tmp.p);
    SP_CHECK_LAUNCH();
    SP_CHECK_CUDA(cudaMemsetAsync(m, 0, V, s));
    std::swap(m, mn);
    int finished = 0;
    SP_TRY(copy_out(&finished, p->tmp.p, sizeof(int), s));
    ++rounds;
    if (finished) break;
    if (rounds > max_rounds) {
      set_error("sp_sssp: no fixed point after %d rounds (negative cycle)", rounds);
      return SP_ERR_NEG_CYCLE;
    }
  }
  if (rounds_out) *rounds_out = rounds;
  if (dist_out) SP_TRY(copy_out(dist_out, p->dist.p, sizeof(int32_t) * V, s));
  return SP_OK;
}

// The schedule of a delta-stepping solve: an explicit delta (argument or sssp.delta
// knob) and the sssp.ctas_per_sm / sssp.local knobs, else the learned choice when a
// model is loaded (cached per weight range and model), else the fixed heuristic.
static int sssp_schedule(sp_graph* g, int64_t& delta, int& ctas, int& local) {
  ctas = g->sssp_ctas_per_sm > 0 ? g->sssp_ctas_per_sm : 4;
  local = g->sssp_local >= 0 ? g->sssp_local : ss::LOCAL_STEPS;
  const int64_t wmax = std::max<int64_t>(1, (int64_t)g->sssp->w_max);
  if (delta <= 0 && g->sssp_delta > 0) delta = g->sssp_delta;
  SsspPlan* sp_ = g->sssp;
  const unsigned gen = mlp_generation();
  if (delta <= 0 && g->sssp_ctas_per_sm == 0 && gen != 0 && sp_->sel_gen == gen && sp_->sel_wmin == sp_->w_min &&
      sp_->sel_wmax == sp_->w_max && sp_->sel_local_knob == g->sssp_local) {
    delta = sp_->sel_delta;  // same inputs as the last scored call
    ctas = sp_->sel_ctas;
    local = sp_->sel_local;
  }
  if (delta <= 0 && g->sssp_ctas_per_sm == 0 && gen != 0) {
    // learned schedule: score every candidate, run the best (fixed heuristic if no
    // model). The cascade budget is a candidate too unless the sssp.local knob is set.
    static const double mults[] = {1, 2, 4, 8, 16, 32, 64};
    static const int cts[] = {1, 2, 4};
    // cascade budgets: off, the default, and a long one (grid 4096^2: 30.8 ms at 64,
    // 28.8 at 256 with the same width and CTAs)
    const int locs[3] = {0, ss::LOCAL_STEPS, 4 * ss::LOCAL_STEPS};
    const int nloc = g->sssp_local >= 0 ? 1 : 3;
    std::vector<float> X;
    struct Cand {
      double mult;
      int ctas, local;
    };
    std::vector<Cand> cand;
    for (double m : mults)
      for (int c : cts)
        for (int l = 0; l < nloc; ++l) {
          const int lv = g->sssp_local >= 0 ? g->sssp_local : locs[l];
          float x[SP_MLP_IN];
          SP_TRY(sssp_features(g, m, c, lv, x));
          X.insert(X.end(), x, x + SP_MLP_IN);
          cand.push_back({m, c, lv});
        }
    std::vector<float> score;
    if (mlp_score(X, score, g->stream) == SP_OK) {
      int best = 0;
      for (int k = 1; k < (int)score.size(); ++k)
        if (score[k] < score[best]) best = k;
      delta = (int64_t)std::llround(cand[best].mult * (double)wmax);
      ctas = cand[best].ctas;
      local = cand[best].local;
      sp_->sel_gen = gen;
      sp_->sel_wmin = sp_->w_min;
      sp_->sel_wmax = sp_->w_max;
      sp_->sel_delta = delta;
      sp_->sel_ctas = ctas;
      sp_->sel_local = local;
      sp_->sel_local_knob = g->sssp_local;
    }
  }
  if (delta <= 0) delta = wmax;
  g->sssp_last_delta = delta;
  g->sssp_last_ctas = ctas;
  g->sssp_last_local = local;
  return SP_OK;
}

int sssp_weights_for(sp_graph* g, const int32_t* weight, const int32_t** w) { return sssp_prepare(g, weight, w); }

int sssp_width_for(sp_graph* g, int64_t& delta) {
  int ctas = 0, local = 0;
  return sssp_schedule(g, delta, ctas, local);
}

int sssp_weight_min(sp_graph* g) { return g->sssp ? g->sssp->w_min : 0; }

}  // namespace sp

extern "C" int sp_sssp(sp_graph_h g, const int32_t* weight, int32_t src, int32_t* dist, int64_t delta,
                       int32_t variant, int32_t* rounds) {
  using namespace sp;
  if (!g || !dist) {
    set_error("sp_sssp: NULL argument");
    return SP_ERR_INVALID;
  }
  if (src < 0 || src >= g->V) {
    set_error("sp_sssp: source %d out of range [0, %d)", src, g->V);
    return SP_ERR_INVALID;
  }
  const int32_t* w = nullptr;
  SP_TRY(sssp_prepare(g, weight, &w));
  if (variant == SP_SSSP_PLAIN) return sssp_plain(g, w, src, dist, rounds);
  if (variant != SP_SSSP_DELTA) {
    set_error("sp_sssp: unknown variant %d", variant);
    return SP_ERR_INVALID;
  }
  int ctas = 0, local = 0;
  SP_TRY(sssp_schedule(g, delta, ctas, local));
  return sssp_delta(g, w, src, dist, delta, ctas, local, rounds);
}

extern "C" int sp_sssp_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                               const int32_t* weight, int32_t source, int32_t* dist) {
  using namespace sp;
  if (!g || !dist || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_sssp_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  if (source < 0 || source >= g->V) {
    set_error("sp_sssp_dynamic: source %d out of range [0, %d)", source, g->V);
    return SP_ERR_INVALID;
  }
  if (!g->has_w) {
    set_error("sp_sssp_dynamic: the graph has no edgeLen");
    return SP_ERR_INVALID;
  }
  bool deletes = false;
  std::vector<int32_t> seeds;
  for (int64_t i = 0; i < n; ++i) {
    if (type[i] == 'd') deletes = true;
    if (type[i] == 'a') seeds.push_back(src[i]);
  }
  // The learned schedule of the last solve carries over the batch when the weights'
  // range is unchanged: scoring again would read the graph's symmetry, which the
  // update forgets (a reverse CSR build on a directed graph).
  struct {
    unsigned gen = 0;
    int wmin = 0, wmax = 0, ctas = 0, local = 0, local_knob = -1;
    int64_t delta = 0;
  } kept;
  if (g->sssp) {
    const SsspPlan* q = g->sssp;
    kept.gen = q->sel_gen;
    kept.wmin = q->sel_wmin;
    kept.wmax = q->sel_wmax;
    kept.ctas = q->sel_ctas;
    kept.local = q->sel_local;
    kept.local_knob = q->sel_local_knob;
    kept.delta = q->sel_delta;
  }
  // A batch with deletions: the parents of the old distances on the old graph (weights
  // >= 1 only, so that they form a forest), and the records on parent edges marked,
  // before the update replaces the graph.
  const int V = g->V;
  cudaStream_t s = g->stream;
  dbuf<int32_t> old_dist, parent, rec;
  dbuf<uint8_t> bad;  // [2 * V]: pointer jumping's two mark buffers
  dbuf<int> nbad;
  bool repair = false;
  g->sssp_last_marked = -1;
  // By default the repair runs on graphs whose last solve from a source took at least
  // REPAIR_MIN_ROUNDS rounds: where a solve takes a dozen rounds (R-MAT 20: 1.3 ms) its
  // fixed passes over the graph cost more than solving again.
  const bool want_repair = g->sssp_repair > 0 || (g->sssp_repair < 0 && g->sssp_last_rounds >= ss::REPAIR_MIN_ROUNDS);
  if (deletes && want_repair) {
    const int32_t* w0 = nullptr;
    SP_TRY(sssp_prepare(g, nullptr, &w0));
    if (g->sssp->w_min >= 1) {
      repair = true;
      SP_TRY(old_dist.alloc(V));
      SP_TRY(parent.alloc(V));
      SP_TRY(bad.alloc(2 * (size_t)V));
      SP_TRY(nbad.alloc(3));
      SP_TRY(rec.alloc(2 * (size_t)std::max<int64_t>(1, n)));
      SP_CHECK_CUDA(cudaMemcpyAsync(old_dist.p, dist, sizeof(int32_t) * V, cudaMemcpyDefault, s));
      ss::k_fill<<<num_sms() * 4, 256, 0, s>>>(V, parent.p, INT_MAX);  // no parent yet
      SP_CHECK_LAUNCH();
      SP_CHECK_CUDA(cudaMemsetAsync(bad.p, 0, V, s));
      SP_CHECK_CUDA(cudaMemsetAsync(nbad.p, 0, 3 * sizeof(int), s));
      SP_CHECK_CUDA(cudaMemcpyAsync(rec.p, src, sizeof(int32_t) * n, cudaMemcpyDefault, s));
      SP_CHECK_CUDA(cudaMemcpyAsync(rec.p + n, dst, sizeof(int32_t) * n, cudaMemcpyDefault, s));
      ss::k_parents<<<num_sms() * 8, 256, 0, s>>>(V, g->off.p, g->adj.p, w0, old_dist.p, parent.p);
      SP_CHECK_LAUNCH();
      ss::k_mark_parent_edges<<<std::max(1, std::min(num_sms() * 4, (int)((n + 255) / 256))), 256, 0, s>>>(
          (int)n, rec.p, rec.p + n, parent.p, V, bad.p, nbad.p);
      SP_CHECK_LAUNCH();
      g_launches += 3;
    }
  }
  int64_t held_adds = 0;
  SP_TRY(update_graph(g, n, type, src, dst, weight, &held_adds));
  g->sssp_last_incremental = 0;
  if (n == 0) return SP_OK;  // nothing changed: the caller's distances stand
  const int32_t* w = nullptr;
  SP_TRY(sssp_prepare(g, nullptr, &w));
  if (kept.gen != 0) {  // sssp_schedule uses it only while model, range and knob match
    SsspPlan* p = g->sssp;
    p->sel_gen = kept.gen;
    p->sel_wmin = kept.wmin;
    p->sel_wmax = kept.wmax;
    p->sel_delta = kept.delta;
    p->sel_ctas = kept.ctas;
    p->sel_local = kept.local;
    p->sel_local_knob = kept.local_knob;
  }
  int64_t delta = 0;
  int ctas = 0, local = 0;
  SP_TRY(sssp_schedule(g, delta, ctas, local));
  if (repair) {
    // DynSSSP's decremental pass (dynamicBatchSSSP:37-60, repair through parents): a
    // marked vertex's subtree loses its support, is reset and lowered again from the
    // unmarked in-neighbours; the solve resumes from those vertices and from the sources
    // of the added edges. Unmarked distances keep a path of unchanged edges, so they stay
    // achievable; only additions can lower them, and the sources of the additions are
    // queued.
    int nb = 0;
    SP_TRY(copy_out(&nb, nbad.p, sizeof(int), s));
    g->sssp_last_marked = 0;
    SsspPlan* p = g->sssp;
    SP_TRY(p->dist.alloc(V));
    SP_CHECK_CUDA(cudaMemcpyAsync(p->dist.p, old_dist.p, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, s));
    std::vector<int32_t> add_src(seeds);
    int nseed = 0;
    dbuf<int32_t> d_seeds, anc;
    SP_TRY(d_seeds.alloc((size_t)V + add_src.size() + 1));
    if (nb > 0) {
      int passes = 1;
      while (passes < 32 && (1ll << (passes - 1)) < (long long)V) ++passes;
      SP_TRY(anc.alloc(2 * (size_t)V));
      ss::k_anc_init<<<num_sms() * 8, 256, 0, s>>>(V, parent.p, anc.p);
      SP_CHECK_LAUNCH();
      int cur = 0;
      for (int k = 0; k < passes; ++k, cur ^= 1) {
        ss::k_jump<<<num_sms() * 8, 256, 0, s>>>(V, anc.p + (size_t)cur * V, bad.p + (size_t)cur * V,
                                                 anc.p + (size_t)(cur ^ 1) * V, bad.p + (size_t)(cur ^ 1) * V);
        SP_CHECK_LAUNCH();
      }
      const uint8_t* marked = bad.p + (size_t)cur * V;
      // a repair that resets more than a quarter of the vertices costs more than a solve
      ss::k_count_marked<<<num_sms() * 4, 256, 0, s>>>(V, marked, nbad.p + 2);
      SP_CHECK_LAUNCH();
      g_launches += (unsigned long long)passes + 2;
      int nmarked = 0;
      SP_TRY(copy_out(&nmarked, nbad.p + 2, sizeof(int), s));
      g->sssp_last_marked = nmarked;
      if ((int64_t)nmarked * 4 > (int64_t)V) return sssp_delta(g, w, source, dist, delta, ctas, local, nullptr);
      ss::k_reset_marked<<<num_sms() * 8, 256, 0, s>>>(V, marked, p->dist.p);
      SP_CHECK_LAUNCH();
      ss::k_push_into_marked<<<num_sms() * 8, 256, 0, s>>>(V, g->off.p, g->adj.p, w, marked, p->dist.p);
      SP_CHECK_LAUNCH();
      ss::k_collect_marked<<<num_sms() * 8, 256, 0, s>>>(V, marked, p->dist.p, d_seeds.p, nbad.p + 1);
      SP_CHECK_LAUNCH();
      g_launches += 3;
      SP_TRY(copy_out(&nseed, nbad.p + 1, sizeof(int), s));
    }
    std::sort(add_src.begin(), add_src.end());
    add_src.erase(std::unique(add_src.begin(), add_src.end()), add_src.end());
    if (!add_src.empty())
      SP_CHECK_CUDA(cudaMemcpyAsync(d_seeds.p + nseed, add_src.data(), sizeof(int32_t) * add_src.size(),
                                    cudaMemcpyHostToDevice, s));
    nseed += (int)add_src.size();
    g->sssp_last_incremental = 2;
    if (nseed == 0) return copy_out(dist, p->dist.p, sizeof(int32_t) * V, s);
    return sssp_delta(g, w, source, dist, delta, ctas, local, nullptr, d_seeds.p, nseed);
  }
  // A deletion (with a weight below 1 somewhere) or an addition of an edge the graph
  // already held (its weight grows by the added weight) can raise distances: solve
  // again from the source.
  if (deletes || held_adds > 0) return sssp_delta(g, w, source, dist, delta, ctas, local, nullptr);
  // additions of new edges only: distances can only drop, and every drop starts at an
  // added edge, so the solve resumes from the old distances with their sources queued
  std::sort(seeds.begin(), seeds.end());
  seeds.erase(std::unique(seeds.begin(), seeds.end()), seeds.end());
  SsspPlan* p = g->sssp;
  SP_TRY(p->dist.alloc(g->V));
  SP_CHECK_CUDA(cudaMemcpyAsync(p->dist.p, dist, sizeof(int32_t) * g->V, cudaMemcpyDefault, s));
  dbuf<int32_t> d_seeds;
  SP_TRY(d_seeds.alloc(seeds.size()));
  SP_CHECK_CUDA(cudaMemcpyAsync(d_seeds.p, seeds.data(), sizeof(int32_t) * seeds.size(), cudaMemcpyHostToDevice, s));
  g->sssp_last_incremental = 1;
  return sssp_delta(g, w, source, dist, delta, ctas, local, nullptr, d_seeds.p, (int)seeds.size());
}

extern "C" int sp_sssp_batch(sp_graph_h g, const int32_t* weight, const int32_t* sources, int32_t nsrc,
                             int32_t* dist) {
  using namespace sp;
  if (!g || !sources || nsrc <= 0 || !dist) {
    set_error("sp_sssp_batch: invalid argument");
    return SP_ERR_INVALID;
  }
  std::vector<int32_t> hs(nsrc);
  SP_TRY(copy_out(hs.data(), sources, sizeof(int32_t) * nsrc, g->stream));
  for (int32_t v : hs)
    if (v < 0 || v >= g->V) {
      set_error("sp_sssp_batch: source %d out of range [0, %d)", v, g->V);
      return SP_ERR_INVALID;
    }
  const int32_t* w = nullptr;
  SP_TRY(sssp_prepare(g, weight, &w));
  int64_t delta = 0;
  int ctas = 0, local = 0;
  SP_TRY(sssp_schedule(g, delta, ctas, local));
  const size_t V = (size_t)g->V;
  return sssp_delta_batches(g, w, hs, delta, ctas, local, [&](const int32_t* rows, int b, int k0) {
    return copy_out(dist + (size_t)k0 * V, rows, sizeof(int32_t) * V * b, g->stream);
  });
}

namespace sp {
// Closeness over weighted distances (sp_centrality.cu): every batch's rows are summed
// on the device, per source, skipping INT_MAX.
int sssp_batch_sums(sp_graph* g, const int32_t* weight, const std::vector<int32_t>& srcs,
                    void (*sum_rows)(const int32_t*, int, int, unsigned long long*, cudaStream_t),
                    unsigned long long* d_sums) {
  const int32_t* w = nullptr;
  SP_TRY(sssp_prepare(g, weight, &w));
  int64_t delta = 0;
  int ctas = 0, local = 0;
  SP_TRY(sssp_schedule(g, delta, ctas, local));
  return sssp_delta_batches(g, w, srcs, delta, ctas, local, [&](const int32_t* rows, int b, int k0) {
    sum_rows(rows, g->V, b, d_sums + k0, g->stream);
    SP_CHECK_LAUNCH();
    return SP_OK;
  });
}
}  // namespace sp

extern "C" int sp_sssp_epoch_trace(sp_graph_h g, float* records, unsigned long long* times, int32_t cap,
                                   int32_t* n) {
  using namespace sp;
  if (!g || !n || cap < 0 || (cap > 0 && (!records || !times))) {
    set_error("sp_sssp_epoch_trace: invalid argument");
    return SP_ERR_INVALID;
  }
  const int have = g->sssp ? g->sssp->etrace_n : 0;
  *n = have;
  const int k = std::min(have, (int)cap);
  if (k == 0) return SP_OK;
  SP_TRY(copy_out(records, g->sssp->etrace.p, sizeof(float) * ss::ETRACE * k, g->stream));
  return copy_out(times, g->sssp->etime.p, sizeof(unsigned long long) * (k + 1), g->stream);
}

extern "C" int sp_sssp_features(sp_graph_h g, const int32_t* weight, double delta_mult, int32_t ctas_per_sm,
                                int32_t local_steps, float* x) {
  using namespace sp;
  if (!g || !x || !(delta_mult > 0) || ctas_per_sm <= 0 || local_steps < 0) {
    set_error("sp_sssp_features: invalid argument");
    return SP_ERR_INVALID;
  }
  const int32_t* w = nullptr;
  SP_TRY(sssp_prepare(g, weight, &w));
  return sssp_features(g, delta_mult, ctas_per_sm, local_steps, x);
}
