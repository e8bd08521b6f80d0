// PageRank that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host engine that hands a plugin its
// device buffers but owns every other byte of GPU memory through its own pool, a
// process working under a hard memory cap, or a latency-critical caller that
// cannot afford the device-wide synchronisation an allocation may cause. For them
// sp_pagerank_noalloc runs the same PageRank (same semantics and tolerance as
// sp_pagerank) on buffers the caller already owns plus a fixed scratch area that
// is part of this library's device image: a file-scope static __device__ array.
// Every GPU that loads the library holds that array (about 12.6 MB) until the
// process exits.
//
// Host code may not use the array's name as a device pointer: on the host it is
// only a stand-in symbol. Its device address is looked up once per device with
// cudaGetSymbolAddress, on the first call made while that device is current;
// that first call should therefore happen before any stream capture. The address
// is kept for the life of the process, so a cudaDeviceReset of a device that has
// made a call is not supported while the library stays loaded. All calls share the
// one array and each call clears what must start at zero, so calls that overlap on
// the GPU (different streams or threads at the same time) race and must be
// serialised by the caller. Each call reads its result state back and synchronises
// its stream before it returns.
//
// The caller's CSR is checked on the device before any gather (offsets start at 0,
// never decrease and end at E; every srcList entry is a vertex id), with the outcome
// kept in the scratch state, so a malformed graph returns SP_ERR_INVALID instead of
// reading outside the caller's arrays.
#include <mutex>

#include "sp_internal.cuh"

namespace sp {
namespace na {

constexpr int MAX_V = 1 << 20;      // largest graph accepted
constexpr int MAX_BLOCKS = 2048;    // per-CTA diff partials
constexpr int THREADS = 256;

struct State {
  int iter;
  int done;
  unsigned int ticket;
  int bad;  // 0, or which check failed: 1 indexofNodes, 2 rev_indexofNodes, 3 srcList
  double diff;
};

// scratch layout: contrib[2][MAX_V] floats, pr_tmp[MAX_V] floats,
// diff_part[MAX_BLOCKS] doubles, one State
constexpr size_t OFF_CONTRIB0 = 0;
constexpr size_t OFF_CONTRIB1 = OFF_CONTRIB0 + sizeof(float) * MAX_V;
constexpr size_t OFF_PRTMP = OFF_CONTRIB1 + sizeof(float) * MAX_V;
constexpr size_t OFF_DIFF = OFF_PRTMP + sizeof(float) * MAX_V;
constexpr size_t OFF_STATE = OFF_DIFF + sizeof(double) * MAX_BLOCKS;
constexpr size_t SCRATCH_BYTES = OFF_STATE + 256;

static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

__global__ void k_init(int V, const int32_t* __restrict__ off, float* __restrict__ pr, float* __restrict__ con,
                       State* st) {
  const float p0 = 1.0f / (float)V;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    pr[v] = p0;
    const int od = off[v + 1] - off[v];
    con[v] = od > 0 ? __fdiv_rn(p0, (float)od) : 0.0f;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->iter = 0;
    st->done = 0;
    st->ticket = 0;
    st->bad = 0;
    st->diff = 0.0;
  }
}

// The caller's CSR, checked before the first iteration (runs after k_init on the same
// stream): a failed check marks the state bad and done, so no iteration gathers.
__global__ void k_check(int V, long long E, const int32_t* __restrict__ off, const int32_t* __restrict__ roff,
                        const int32_t* __restrict__ radj, State* st) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int bad = 0;
  for (long long v = tid; v <= V; v += stride) {
    const int a = off[v], b = roff[v];
    if (v == 0 ? a != 0 : a < off[v - 1]) bad = 1;
    if (v == V && a != E) bad = 1;
    if (v == 0 ? b != 0 : b < roff[v - 1]) bad = 2;
    if (v == V && b != E) bad = 2;
  }
  for (long long e = tid; e < E; e += stride) {
    const int u = radj[e];
    if (u < 0 || u >= V) bad = 3;
  }
  if (bad) {
    atomicMax(&st->bad, bad);
    st->done = 1;
  }
}

// One iteration: a warp per row (lanes over in-edges, FP64 partials, fixed xor
// tree), per-CTA diff partials summed in CTA order by the last CTA to finish.
__global__ void __launch_bounds__(THREADS) k_iter(int V, const int32_t* __restrict__ off,
                                                  const int32_t* __restrict__ roff, const int32_t* __restrict__ radj,
                                                  const float* __restrict__ pr_old, const float* __restrict__ con_old,
                                                  float* __restrict__ pr_new, float* __restrict__ con_new,
                                                  double* diff_part, State* st, float base, float delta, double beta,
                                                  int max_iter) {
  __shared__ double s_red[THREADS / 32];
  __shared__ int s_last;
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  double my_diff = 0;
  for (int r = (blockIdx.x * THREADS + threadIdx.x) >> 5; r < V; r += (gridDim.x * THREADS) >> 5) {
    double acc = 0;
    for (int e = roff[r] + lane; e < roff[r + 1]; e += 32) acc += (double)__ldg(con_old + __ldg(radj + e));
    acc = warp_sum(acc);
    if (lane == 0) {
      const float np = __fadd_rn(base, __fmul_rn(delta, (float)acc));
      const int od = off[r + 1] - off[r];
      my_diff += fabs((double)np - (double)pr_old[r]);
      pr_new[r] = np;
      con_new[r] = od > 0 ? __fdiv_rn(np, (float)od) : 0.0f;
    }
  }
  const double bd = block_sum<THREADS>(my_diff, s_red);
  if (threadIdx.x == 0) {
    diff_part[blockIdx.x] = bd;
    __threadfence();
    s_last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const volatile double* dp = diff_part;
    double p = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += THREADS) p += dp[i];
    const double total = block_sum<THREADS>(p, s_red);
    if (threadIdx.x == 0) {
      const int it = st->iter + 1;
      st->iter = it;
      st->diff = total;
      st->done = (total > beta && it < max_iter) ? 0 : 1;
      st->ticket = 0;
    }
  }
}

std::mutex g_mu;
void* g_addr[128] = {};  // scratch device address per device ordinal

}  // namespace na
}  // namespace sp

using namespace sp;

extern "C" int sp_pagerank_noalloc(const int32_t* indexofNodes, const int32_t* rev_indexofNodes,
                                   const int32_t* srcList, int32_t V, int64_t E, float beta, float delta,
                                   int32_t maxIter, float* pageRank, int32_t* iterations, void* cuda_stream) {
  if (V <= 0 || V > na::MAX_V) {
    set_error("sp_pagerank_noalloc: V = %d is outside 1..%d (the fixed scratch holds %d vertices)", V, na::MAX_V,
              na::MAX_V);
    return SP_ERR_INVALID;
  }
  if (E < 0 || E >= (int64_t)INT32_MAX || !indexofNodes || !rev_indexofNodes || (E > 0 && !srcList) || !pageRank) {
    set_error("sp_pagerank_noalloc: invalid argument (device CSR pointers and output are required)");
    return SP_ERR_INVALID;
  }
  int dev = 0;
  SP_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) {
    set_error("sp_pagerank_noalloc: device ordinal %d not supported", dev);
    return SP_ERR_UNSUPPORTED;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(na::g_mu);
    if (!na::g_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, na::g_scratch);
      if (e != cudaSuccess) {
        set_error("sp_pagerank_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return SP_ERR_CUDA;
      }
      na::g_addr[dev] = p;
    }
    base = static_cast<unsigned char*>(na::g_addr[dev]);
  }
  cudaStream_t s = (cudaStream_t)cuda_stream;
  float* con[2] = {reinterpret_cast<float*>(base + na::OFF_CONTRIB0), reinterpret_cast<float*>(base + na::OFF_CONTRIB1)};
  float* pr[2] = {pageRank, reinterpret_cast<float*>(base + na::OFF_PRTMP)};
  double* diff_part = reinterpret_cast<double*>(base + na::OFF_DIFF);
  na::State* st = reinterpret_cast<na::State*>(base + na::OFF_STATE);
  const int n_iter = maxIter > 0 ? maxIter : 1;  // the DSL's do-while runs the body at least once
  const float fbase = (1.0f - delta) / (float)V;
  const int grid = std::min(na::MAX_BLOCKS, num_sms() * 8);
  na::k_init<<<num_sms() * 4, na::THREADS, 0, s>>>(V, indexofNodes, pr[0], con[0], st);
  SP_CHECK_LAUNCH();
  na::k_check<<<num_sms() * 4, na::THREADS, 0, s>>>(V, (long long)E, indexofNodes, rev_indexofNodes, srcList, st);
  SP_CHECK_LAUNCH();
  for (int k = 0; k < n_iter; ++k) {
    const int c = k & 1, n = c ^ 1;
    na::k_iter<<<grid, na::THREADS, 0, s>>>(V, indexofNodes, rev_indexofNodes, srcList, pr[c], con[c], pr[n], con[n],
                                           diff_part, st, fbase, delta, (double)beta, n_iter);
    SP_CHECK_LAUNCH();
  }
  na::State hs;
  SP_CHECK_CUDA(cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
  SP_CHECK_CUDA(cudaStreamSynchronize(s));
  if (hs.bad) {
    static const char* what[] = {"", "indexofNodes (must start at 0, never decrease and end at E)",
                                 "rev_indexofNodes (must start at 0, never decrease and end at E)",
                                 "srcList (every entry must be a vertex id in [0, V))"};
    set_error("sp_pagerank_noalloc: malformed %s; no ranks were computed", what[hs.bad & 3]);
    return SP_ERR_INVALID;
  }
  if (hs.iter & 1) {  // the last iteration wrote the scratch copy
    SP_CHECK_CUDA(cudaMemcpyAsync(pageRank, pr[1], sizeof(float) * V, cudaMemcpyDeviceToDevice, s));
    SP_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  if (iterations) *iterations = hs.iter;
  return SP_OK;
}
