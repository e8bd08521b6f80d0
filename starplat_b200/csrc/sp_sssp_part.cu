// Single-source SSSP split over GPUs by vertices: the 1-D vertex partition with a
// per-bucket frontier exchange. It replaces the host-staged property copies of the
// reference's multi-GPU generator (backend_multigpu/dsl_cpp_generator.cpp:604-678,
// :964-1005) for Compute_SSSP (staticDSLCodes/sssp_dslV3:1-26).
//
// Every rank holds the whole graph and owns the vertices v with v % nparts == part.
// dist[v] is authoritative only for owned v (the other entries stay INT_MAX). A solve
// is delta-stepping in bulk-synchronous rounds, driven by the caller:
//   relax    the owned frontier's out-edges. A candidate for an owned target lowers
//            dist with atomicMin and queues the target: into the next round's frontier
//            below the bucket end, else into the far pile. A candidate for another
//            part's vertex lowers a per-round outbox entry obox[u] and, the first time
//            in the round, appends u to that part's send region. So each part receives
//            at most one message per vertex per round: (u, the smallest candidate).
//            The regions are packed in part order into the caller's send buffer.
//            Frontier vertices with more than HUB_DEG out-edges are relaxed in pieces
//            shared by all warps.
//   (the caller's all-to-all moves the messages; NCCL on device buffers)
//   apply    the received messages, like local candidates; the new frontier's size
//            goes to the caller, who sums it over the ranks.
//   far_min / advance: when no rank has a frontier, the smallest far distance (the
//            caller takes the minimum over the ranks) sets the next bucket end, and
//            each far pile is split into the new frontier and the rest.
// Mark bitmaps: the next frontier's marks alternate between two bitmaps by round
// parity (the current frontier's marks are cleared as it is read), the far pile's by
// epoch parity (cleared at the split), and the outbox marks are cleared by the pack.
// Every vertex enters a queue at most once per round or epoch, so the queues hold at
// most the part's owned vertices. Appends are bounds-checked anyway: an overflow or a
// message for a vertex this part does not own sets a status bit, which the next call
// reports as an error.
// Negative weights: one bucket (Bellman-Ford rounds), bounded by 4V + 64 rounds; a
// longer run means a reachable negative cycle (SP_ERR_NEG_CYCLE), as in sp_sssp.
#include <climits>

#include "sp_internal.cuh"

namespace sp {
namespace ssp {

constexpr int THREADS = 256;
constexpr unsigned FULL = 0xffffffffu;
constexpr long long NO_BUCKETS = 1ll << 62;  // bucket width for negative weights
// Frontier vertices above HUB_DEG out-edges are relaxed in HUB_CHUNK-edge pieces that
// all warps share (a second kernel), so no warp walks an R-MAT hub's row alone.
constexpr int HUB_DEG = 1024;
constexpr int HUB_CHUNK = 256;

struct Ctl {
  int qcount[2];       // frontier entries by round parity
  int fcount[2];       // far-pile entries by epoch parity
  int status;          // 1: an append past a bound; 2: a message for a vertex not owned here
  int pad;
  unsigned long long hcount;  // this round's hub entries (high 32 bits) and their pieces (low)
  long long thr;       // end of the current bucket
  long long thr_old;   // end of the previous bucket (for the split)
};

struct Args {
  const int32_t* __restrict__ off;
  const int32_t* __restrict__ adj;
  const int32_t* __restrict__ w;
  int32_t* dist;
  int32_t* obox;
  const int32_t* Q;    // this round's frontier
  int32_t* QN;         // the next round's frontier
  int32_t* F;          // this epoch's far pile
  unsigned* qcur;      // marks of Q (cleared as Q is read)
  unsigned* qnext;     // marks of QN
  unsigned* fbits;     // marks of F
  unsigned* sbits;     // outbox marks
  int32_t* region;     // [np][cap] vertex ids per destination part
  int32_t* rcount;     // [np] entries per region
  int32_t* hv;         // this round's hub vertices
  int32_t* hb;         // first piece of each hub entry (increasing with the entry)
  Ctl* ctl;
  int np, part, V, cap, round, epoch;
};

__device__ __forceinline__ bool mark(unsigned* bm, int u) {
  const unsigned b = 1u << (u & 31);
  return (atomicOr(bm + (u >> 5), b) & b) == 0u;
}

__device__ __forceinline__ void unmark(unsigned* bm, int u) { atomicAnd(bm + (u >> 5), ~(1u << (u & 31))); }

__device__ __forceinline__ void append(Ctl* ctl, int32_t* buf, int* counter, int cap, int val) {
  const int i = atomicAdd(counter, 1);
  if (i < cap)
    buf[i] = val;
  else
    atomicOr(&ctl->status, 1);
}

// An owned vertex u reached with candidate nd (already known to lower dist[u]).
__device__ __forceinline__ void queue_owned(const Args& a, int u, long long nd, long long thr) {
  if (nd < thr) {
    if (mark(a.qnext, u)) append(a.ctl, a.QN, &a.ctl->qcount[(a.round + 1) & 1], a.cap, u);
  } else {
    if (mark(a.fbits, u)) append(a.ctl, a.F, &a.ctl->fcount[a.epoch & 1], a.cap, u);
  }
}

__device__ __forceinline__ void relax_one(const Args& a, int u, long long nd, long long thr) {
  const int r = u % a.np;
  if (r == a.part) {
    const int old = atomicMin(a.dist + u, (int)nd);
    if (nd < (long long)old) queue_owned(a, u, nd, thr);
  } else {
    const int old = atomicMin(a.obox + u, (int)nd);
    if (nd < (long long)old && mark(a.sbits, u))
      append(a.ctl, a.region + (size_t)r * a.cap, a.rcount + r, a.cap, u);
  }
}

// dist = obox = INT_MAX everywhere; the counters and the bucket end reset.
__global__ void k_init(int V, int32_t* dist, int32_t* obox, Ctl* ctl, long long delta) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    dist[v] = INT_MAX;
    obox[v] = INT_MAX;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->qcount[0] = ctl->qcount[1] = 0;
    ctl->fcount[0] = ctl->fcount[1] = 0;
    ctl->status = 0;
    ctl->hcount = 0ull;
    ctl->thr = delta;
    ctl->thr_old = 0;
  }
}

__global__ void k_seed(int src, int np, int part, int32_t* dist, int32_t* q0, Ctl* ctl) {
  if (src % np == part) {
    dist[src] = 0;
    q0[0] = src;
    ctl->qcount[0] = 1;
  }
}

// One round: warps take 32 frontier vertices at a time; their edges are flattened over
// the warp's lanes (an exclusive scan of the degrees), 32 edges per step.
__global__ void __launch_bounds__(THREADS) k_relax(Args a) {
  const int lane = threadIdx.x & 31;
  const int nq = min(a.ctl->qcount[a.round & 1], a.cap);
  const long long thr = a.ctl->thr;
  const int gw = (blockIdx.x * THREADS + threadIdx.x) >> 5, nw = (gridDim.x * THREADS) >> 5;
  for (int base = gw * 32; base < nq; base += nw * 32) {
    const int i = base + lane;
    int v = -1, b = 0, d = 0;
    long long dv = 0;
    if (i < nq) {
      v = a.Q[i];
      unmark(a.qcur, v);
      b = a.off[v];
      d = a.off[v + 1] - b;
      dv = __ldcg(a.dist + v);
      if (d > HUB_DEG) {  // its pieces go to k_relax_hubs; the entry and piece base together
        const unsigned long long nch = (unsigned)((d + HUB_CHUNK - 1) / HUB_CHUNK);
        const unsigned long long old = atomicAdd(&a.ctl->hcount, (1ull << 32) | nch);
        const int h = (int)(old >> 32);
        if (h < a.cap) {
          a.hv[h] = v;
          a.hb[h] = (int)(old & 0xffffffffull);
        } else {
          atomicOr(&a.ctl->status, 1);
        }
        d = 0;
      }
    }
    int inc = d;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
      const int t = __shfl_up_sync(FULL, inc, k);
      if (lane >= k) inc += t;
    }
    const int total = __shfl_sync(FULL, inc, 31);
    const int excl = inc - d;
    for (int t0 = 0; t0 < total; t0 += 32) {
      const int t = t0 + lane;
      int j = 0;  // the last lane whose edges start at or before t
#pragma unroll
      for (int k = 16; k > 0; k >>= 1)
        if (__shfl_sync(FULL, excl, j + k) <= t) j += k;
      const int jb = __shfl_sync(FULL, b, j);
      const int je = __shfl_sync(FULL, excl, j);
      const long long jd = __shfl_sync(FULL, dv, j);
      if (t < total) {
        const int k = jb + (t - je);
        const long long nd = jd + (long long)a.w[k];
        if (nd < (long long)INT_MAX) relax_one(a, a.adj[k], nd, thr);
      }
    }
  }
}

// The hub pieces of this round, a warp per piece: the entry is the last one whose
// first piece is at or below the piece's index.
__global__ void __launch_bounds__(THREADS) k_relax_hubs(Args a) {
  const int lane = threadIdx.x & 31;
  const unsigned long long hc = a.ctl->hcount;
  const int nh = min((int)(hc >> 32), a.cap);
  const int pieces = nh > 0 ? (int)(hc & 0xffffffffull) : 0;
  const long long thr = a.ctl->thr;
  const int gw = (blockIdx.x * THREADS + threadIdx.x) >> 5, nw = (gridDim.x * THREADS) >> 5;
  for (int ch = gw; ch < pieces; ch += nw) {
    int lo = 0, hi = nh - 1;
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (a.hb[m] <= ch) lo = m; else hi = m - 1;
    }
    const int v = a.hv[lo];
    const long long dv = __ldcg(a.dist + v);
    const int vb = a.off[v] + (ch - a.hb[lo]) * HUB_CHUNK;
    const int ve = min(vb + HUB_CHUNK, a.off[v + 1]);
    for (int k = vb + lane; k < ve; k += 32) {
      const long long nd = dv + (long long)a.w[k];
      if (nd < (long long)INT_MAX) relax_one(a, a.adj[k], nd, thr);
    }
  }
}

// Packs the regions in part order into send (pairs u, obox[u]) and resets the outbox
// entries and marks they used. Block row y = destination part.
__global__ void k_pack(Args a, int32_t* __restrict__ send, int32_t* __restrict__ send_counts) {
  const int r = blockIdx.y;
  int at = 0;
  for (int q = 0; q < r; ++q) at += min(a.rcount[q], a.cap);
  const int n = min(a.rcount[r], a.cap);
  const int32_t* reg = a.region + (size_t)r * a.cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int u = reg[i];
    send[2 * (size_t)(at + i)] = u;
    send[2 * (size_t)(at + i) + 1] = a.obox[u];
    a.obox[u] = INT_MAX;
    unmark(a.sbits, u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) send_counts[r] = n;
}

// Received (u, d) pairs: owned targets only, like local candidates.
__global__ void __launch_bounds__(THREADS) k_apply(Args a, const int32_t* __restrict__ msg, int n) {
  const long long thr = a.ctl->thr;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int u = msg[2 * (size_t)i], d = msg[2 * (size_t)i + 1];
    if (u < 0 || u >= a.V || u % a.np != a.part) {
      atomicOr(&a.ctl->status, 2);
      continue;
    }
    const int old = atomicMin(a.dist + u, d);
    if (d < old) queue_owned(a, u, d, thr);
  }
}

// End of round k: its frontier's count and hub list are consumed; the next frontier's
// size goes out.
__global__ void k_round_end(Ctl* ctl, int round, int cap, int32_t* frontier) {
  ctl->qcount[round & 1] = 0;
  ctl->hcount = 0ull;
  *frontier = min(ctl->qcount[(round + 1) & 1], cap);
}

__global__ void k_far_init(int32_t* out) { *out = INT_MAX; }

// The smallest distance in the far pile at or above the current bucket end (entries
// lowered below it since were relaxed in this bucket).
__global__ void k_far_min(const int32_t* __restrict__ F, const Ctl* ctl, int epoch, int cap,
                          const int32_t* __restrict__ dist, int32_t* out) {
  const int n = min(ctl->fcount[epoch & 1], cap);
  const long long thr = ctl->thr;
  int m = INT_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int d = __ldcg(dist + F[i]);
    if ((long long)d >= thr) m = min(m, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(FULL, m, o));
  if ((threadIdx.x & 31) == 0 && m != INT_MAX) atomicMin(out, m);
}

// Next bucket: the one holding the smallest far distance over all parts.
__global__ void k_bucket(Ctl* ctl, const int32_t* far_min, long long delta) {
  const long long fm = *far_min;
  ctl->thr_old = ctl->thr;
  ctl->thr = (fm / delta + 1) * delta;
}

// Far pile of the previous epoch -> the frontier of the coming round (below the new
// bucket end; that round's queue and marks, which the round reads and clears) or the
// new epoch's far pile; entries settled in earlier buckets are dropped. a.epoch is the
// new epoch, a.round the coming round (whose frontier is empty on every part).
__global__ void k_split(Args a, const int32_t* __restrict__ Fin, unsigned* fin_bits) {
  const int n = min(a.ctl->fcount[(a.epoch + 1) & 1], a.cap);
  const long long thr_old = a.ctl->thr_old, thr = a.ctl->thr;
  int32_t* Q = const_cast<int32_t*>(a.Q);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int u = Fin[i];
    unmark(fin_bits, u);
    const long long d = __ldcg(a.dist + u);
    if (d < thr_old) continue;
    if (d < thr) {
      if (mark(a.qcur, u)) append(a.ctl, Q, &a.ctl->qcount[a.round & 1], a.cap, u);
    } else {
      if (mark(a.fbits, u)) append(a.ctl, a.F, &a.ctl->fcount[a.epoch & 1], a.cap, u);
    }
  }
}

__global__ void k_split_end(Ctl* ctl, int round, int epoch, int cap, int32_t* frontier) {
  ctl->fcount[(epoch + 1) & 1] = 0;  // the previous epoch's pile is consumed
  *frontier = min(ctl->qcount[round & 1], cap);
}

}  // namespace ssp

struct SsspPartPlan {
  int part = 0, np = 1, V = 0, cap = 0, nwords = 0;
  int round = 0, epoch = 0;
  long long delta = 1;
  long long max_rounds = 0;
  const int32_t* w = nullptr;
  dbuf<int32_t> dist, obox, q[2], f[2], region, rcount, hv, hb;
  dbuf<unsigned> bits;  // qbits[2], fbits[2], sbits
  dbuf<ssp::Ctl> ctl;
};

void free_sssp_part_plan(SsspPartPlan* p) { delete p; }

static ssp::Args part_args(sp_graph* g, SsspPartPlan* p) {
  ssp::Args a;
  a.off = g->off.p;
  a.adj = g->adj.p;
  a.w = p->w;
  a.dist = p->dist.p;
  a.obox = p->obox.p;
  a.Q = p->q[p->round & 1].p;
  a.QN = p->q[(p->round + 1) & 1].p;
  a.F = p->f[p->epoch & 1].p;
  a.qcur = p->bits.p + (size_t)(p->round & 1) * p->nwords;
  a.qnext = p->bits.p + (size_t)((p->round + 1) & 1) * p->nwords;
  a.fbits = p->bits.p + (size_t)(2 + (p->epoch & 1)) * p->nwords;
  a.sbits = p->bits.p + (size_t)4 * p->nwords;
  a.region = p->region.p;
  a.rcount = p->rcount.p;
  a.hv = p->hv.p;
  a.hb = p->hb.p;
  a.ctl = p->ctl.p;
  a.np = p->np;
  a.part = p->part;
  a.V = p->V;
  a.cap = p->cap;
  a.round = p->round;
  a.epoch = p->epoch;
  return a;
}

// The plan of a begun split solve, and no flagged status (which stops the solve).
static int part_plan(sp_graph* g, const char* who, SsspPartPlan** out) {
  if (!g || !g->sssp_part || !g->sssp_part->ctl.p) {
    set_error("%s: no split SSSP begun on this graph", who);
    return SP_ERR_INVALID;
  }
  *out = g->sssp_part;
  return SP_OK;
}

static int part_status(sp_graph* g, SsspPartPlan* p, const char* who) {
  int st = 0;
  SP_TRY(copy_out(&st, &p->ctl.p->status, sizeof(int), g->stream));
  if (st & 2) {
    set_error("%s: a received message names a vertex this part does not own", who);
    return SP_ERR_INVALID;
  }
  if (st) {
    set_error("%s: a queue append went past its bound", who);
    return SP_ERR_CUDA;
  }
  return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" int sp_sssp_part_begin(sp_graph_h g, int32_t part, int32_t nparts, const int32_t* weight, int32_t src,
                                  int64_t delta, int32_t* cap) {
  if (!g || nparts < 1 || part < 0 || part >= nparts || !cap) {
    set_error("sp_sssp_part_begin: invalid argument");
    return SP_ERR_INVALID;
  }
  if (src < 0 || src >= g->V) {
    set_error("sp_sssp_part_begin: source %d out of range [0, %d)", src, g->V);
    return SP_ERR_INVALID;
  }
  const int32_t* w = nullptr;
  SP_TRY(sssp_weights_for(g, weight, &w));
  if (sssp_weight_min(g) < 0) {
    delta = ssp::NO_BUCKETS;
  } else if (delta <= 0) {
    SP_TRY(sssp_width_for(g, delta));
  }
  if (!g->sssp_part) g->sssp_part = new SsspPartPlan();
  SsspPartPlan* p = g->sssp_part;
  const int V = g->V;
  p->part = part;
  p->np = nparts;
  p->V = V;
  p->cap = (V + nparts - 1) / nparts;  // owned vertices of any part
  p->nwords = (V + 31) / 32;
  p->round = 0;
  p->epoch = 0;
  p->delta = std::max<long long>(1, delta);
  p->max_rounds = 4ll * V + 64;
  p->w = w;
  SP_TRY(p->dist.alloc(V));
  SP_TRY(p->obox.alloc(V));
  for (int k = 0; k < 2; ++k) {
    SP_TRY(p->q[k].alloc(p->cap));
    SP_TRY(p->f[k].alloc(p->cap));
  }
  SP_TRY(p->region.alloc((size_t)nparts * p->cap));
  SP_TRY(p->rcount.alloc(nparts));
  SP_TRY(p->hv.alloc(p->cap));
  SP_TRY(p->hb.alloc(p->cap));
  SP_TRY(p->bits.alloc((size_t)5 * p->nwords));
  SP_TRY(p->ctl.alloc(1));
  cudaStream_t s = g->stream;
  SP_CHECK_CUDA(cudaMemsetAsync(p->bits.p, 0, sizeof(unsigned) * 5 * (size_t)p->nwords, s));
  ssp::k_init<<<num_sms() * 4, 256, 0, s>>>(V, p->dist.p, p->obox.p, p->ctl.p, p->delta);
  SP_CHECK_LAUNCH();
  ssp::k_seed<<<1, 1, 0, s>>>(src, nparts, part, p->dist.p, p->q[0].p, p->ctl.p);
  SP_CHECK_LAUNCH();
  g_launches += 2;
  *cap = p->cap;
  return SP_OK;
}

extern "C" int sp_sssp_part_relax(sp_graph_h g, int32_t* send, int32_t* send_counts) {
  SsspPartPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_sssp_part_relax", &p));
  if (!send || !send_counts) {
    set_error("sp_sssp_part_relax: NULL buffer");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  SP_CHECK_CUDA(cudaMemsetAsync(p->rcount.p, 0, sizeof(int32_t) * p->np, s));
  const ssp::Args a = part_args(g, p);
  ssp::k_relax<<<num_sms() * 8, ssp::THREADS, 0, s>>>(a);
  SP_CHECK_LAUNCH();
  ssp::k_relax_hubs<<<num_sms() * 8, ssp::THREADS, 0, s>>>(a);
  SP_CHECK_LAUNCH();
  ssp::k_pack<<<dim3(std::max(1, std::min(num_sms() * 2, (p->cap + 255) / 256)), p->np), 256, 0, s>>>(a, send,
                                                                                                       send_counts);
  SP_CHECK_LAUNCH();
  g_launches += 3;
  return SP_OK;
}

extern "C" int sp_sssp_part_apply(sp_graph_h g, const int32_t* msgs, int32_t n, int32_t* frontier) {
  SsspPartPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_sssp_part_apply", &p));
  if (n < 0 || (n > 0 && !msgs) || !frontier || (int64_t)n > (int64_t)p->np * p->cap) {
    set_error("sp_sssp_part_apply: invalid argument");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  const ssp::Args a = part_args(g, p);
  if (n > 0) {
    ssp::k_apply<<<std::max(1, std::min(num_sms() * 4, (n + 255) / 256)), ssp::THREADS, 0, s>>>(a, msgs, n);
    SP_CHECK_LAUNCH();
    g_launches += 1;
  }
  ssp::k_round_end<<<1, 1, 0, s>>>(p->ctl.p, p->round, p->cap, frontier);
  SP_CHECK_LAUNCH();
  g_launches += 1;
  ++p->round;
  if ((long long)p->round > p->max_rounds) {
    set_error("sp_sssp_part_apply: more than %lld rounds: a negative cycle is reachable from the source",
              p->max_rounds);
    return SP_ERR_NEG_CYCLE;
  }
  if ((p->round & 63) == 0) SP_TRY(part_status(g, p, "sp_sssp_part_apply"));
  return SP_OK;
}

extern "C" int sp_sssp_part_far_min(sp_graph_h g, int32_t* far_min) {
  SsspPartPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_sssp_part_far_min", &p));
  if (!far_min) {
    set_error("sp_sssp_part_far_min: NULL buffer");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  ssp::k_far_init<<<1, 1, 0, s>>>(far_min);
  SP_CHECK_LAUNCH();
  ssp::k_far_min<<<std::max(1, std::min(num_sms() * 4, (p->cap + 255) / 256)), 256, 0, s>>>(
      p->f[p->epoch & 1].p, p->ctl.p, p->epoch, p->cap, p->dist.p, far_min);
  SP_CHECK_LAUNCH();
  g_launches += 2;
  return SP_OK;
}

extern "C" int sp_sssp_part_advance(sp_graph_h g, const int32_t* far_min, int32_t* frontier) {
  SsspPartPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_sssp_part_advance", &p));
  if (!far_min || !frontier) {
    set_error("sp_sssp_part_advance: NULL buffer");
    return SP_ERR_INVALID;
  }
  cudaStream_t s = g->stream;
  ssp::k_bucket<<<1, 1, 0, s>>>(p->ctl.p, far_min, p->delta);
  SP_CHECK_LAUNCH();
  const int32_t* Fin = p->f[p->epoch & 1].p;
  unsigned* fin_bits = p->bits.p + (size_t)(2 + (p->epoch & 1)) * p->nwords;
  ++p->epoch;  // the split fills the new epoch's pile
  const ssp::Args a = part_args(g, p);
  ssp::k_split<<<std::max(1, std::min(num_sms() * 4, (p->cap + 255) / 256)), 256, 0, s>>>(a, Fin, fin_bits);
  SP_CHECK_LAUNCH();
  ssp::k_split_end<<<1, 1, 0, s>>>(p->ctl.p, p->round, p->epoch, p->cap, frontier);
  SP_CHECK_LAUNCH();
  g_launches += 3;
  return SP_OK;
}

extern "C" int sp_sssp_part_dist(sp_graph_h g, int32_t* dist) {
  SsspPartPlan* p = nullptr;
  SP_TRY(part_plan(g, "sp_sssp_part_dist", &p));
  if (!dist) {
    set_error("sp_sssp_part_dist: NULL buffer");
    return SP_ERR_INVALID;
  }
  SP_TRY(part_status(g, p, "sp_sssp_part_dist"));
  return copy_out(dist, p->dist.p, sizeof(int32_t) * (size_t)p->V, g->stream);
}
