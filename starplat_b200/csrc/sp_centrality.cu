// Degree and closeness centrality for sm_100a, on the SSSP and BFS kernels.
//
// Semantics:
//  * Degree (staticDSLCodes/degree_centrality:1-6): deg[v] = count_outNbrs(v), the
//    out-degree indexofNodes[v+1] - indexofNodes[v] (backend_omp/dsl_cpp_generator.cpp:2475-2484).
//  * Compute_CC (staticDSLCodes/CC:1-26): for every source, the fixedPoint Min
//    relaxation converges to the shortest-path distances over the edge weights;
//    temp = the sum of the finite ones; CC[src] = 1.0 / temp, every other vertex 0.
//    The distances come from the batched delta-stepping kernel (sp_sssp_batch: one
//    cooperative launch runs a batch of sources, each on its own group of CTAs, with
//    the learned schedule) and the sum from a device reduction in 64 bits: the DSL's int temp overflows past
//    2^31 - 1, and the exact sum is reported instead.
//  * Compute_CC_Unweighted (staticDSLCodes/closeness_centrality_unwt:1-20): dist
//    starts at 0 and iterateInBFS sets w.dist = v.dist + 1 for next-level neighbours
//    only (the generator's bfsDist guard, backend_omp/dsl_cpp_generator.cpp:1461-1468),
//    so dist is the BFS level of every reached vertex and 0 elsewhere; CC[src] =
//    1.0 / the sum of dist. The levels come from the forward pass of the batched BC
//    kernel, 64 sources per pass.
// 1.0 / sum is a double division stored as float, as the generated C++ computes it
// (a zero sum gives +inf). Sources are a set in the DSL: they must be distinct.
#include <algorithm>
#include <cmath>
#include <vector>

#include "sp_internal.cuh"

namespace sp {

// Levels (-1 = unreached) and path counts of up to 64 sources, source-major (sp_bc.cu).
int bc_levels(sp_graph* g, const int32_t* d_srcs, int nsrc, int32_t* lvl_out, double* sig_out);
// Batched delta-stepping (sp_sssp.cu): the distance rows of every batch go to sum_rows.
int sssp_batch_sums(sp_graph* g, const int32_t* weight, const std::vector<int32_t>& srcs,
                    void (*sum_rows)(const int32_t*, int, int, unsigned long long*, cudaStream_t),
                    unsigned long long* d_sums);

namespace cen {

__global__ void k_outdeg(const int32_t* __restrict__ off, int V, int32_t* __restrict__ deg) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) deg[v] = off[v + 1] - off[v];
}

// Per source k < nsrc: out[k] += sum of d[k * V + v] over v with d[k * V + v] != skip
// (64-bit two's complement, so negative distances add correctly).
__global__ void k_sum_except(const int32_t* __restrict__ d, int V, int nsrc, int32_t skip,
                             unsigned long long* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  for (int k = 0; k < nsrc; ++k) {
    const int32_t* row = d + (size_t)k * V;
    long long s = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
      const int32_t x = row[v];
      if (x != skip) s += x;
    }
    s = warp_sum(s);
    if (lane == 0 && s != 0) atomicAdd(out + k, (unsigned long long)s);
  }
}

// Sums of the finite distances of b source-major rows (the batched SSSP callback).
void sum_finite_rows(const int32_t* rows, int V, int b, unsigned long long* out, cudaStream_t s) {
  k_sum_except<<<num_sms() * 4, 256, 0, s>>>(rows, V, b, INT32_MAX, out);
}

}  // namespace cen

// Sources as a host vector: range-checked and distinct.
static int read_sources(sp_graph* g, const int32_t* sources, int32_t nsrc, std::vector<int32_t>& hs,
                        const char* who) {
  hs.resize(nsrc);
  SP_TRY(copy_out(hs.data(), sources, sizeof(int32_t) * nsrc, g->stream));
  std::vector<int32_t> u = hs;
  std::sort(u.begin(), u.end());
  if (std::adjacent_find(u.begin(), u.end()) != u.end() || u.front() < 0 || u.back() >= g->V) {
    set_error("%s: sources must be distinct vertices in [0, %d)", who, g->V);
    return SP_ERR_INVALID;
  }
  return SP_OK;
}

// CC[V] = 0 except CC[src_k] = 1.0 / sums[k], written to a host or device array.
static int write_closeness(sp_graph* g, const std::vector<int32_t>& hs, const std::vector<long long>& sums,
                           float* CC) {
  std::vector<float> out(g->V, 0.0f);
  for (size_t k = 0; k < hs.size(); ++k) out[hs[k]] = (float)(1.0 / (double)sums[k]);
  if (g->V == 0) return SP_OK;
  SP_CHECK_CUDA(cudaMemcpyAsync(CC, out.data(), sizeof(float) * g->V, cudaMemcpyDefault, g->stream));
  SP_CHECK_CUDA(cudaStreamSynchronize(g->stream));
  return SP_OK;
}

}  // namespace sp

extern "C" int sp_degree_centrality(sp_graph_h g, int32_t* deg) {
  using namespace sp;
  if (!g || !deg) {
    set_error("sp_degree_centrality: NULL argument");
    return SP_ERR_INVALID;
  }
  if (g->V == 0) return SP_OK;
  dbuf<int32_t> d;
  SP_TRY(d.alloc(g->V));
  cen::k_outdeg<<<num_sms() * 4, 256, 0, g->stream>>>(g->off.p, g->V, d.p);
  SP_CHECK_LAUNCH();
  return copy_out(deg, d.p, sizeof(int32_t) * g->V, g->stream);
}

// DynDegree's Batch block (dynamicDSLCodes/dynamicBatchDeg:26-37): the batch, then the
// out-degrees of the updated graph. The DSL adjusts deg[src] by one per update, which
// also counts deletions of absent edges and additions of present ones; the degrees here
// are read from the updated rows, so they are exact.
extern "C" int sp_degree_dynamic(sp_graph_h g, int64_t n, const char* type, const int32_t* src, const int32_t* dst,
                                 const int32_t* weight, int32_t* deg) {
  using namespace sp;
  if (!g || !deg || n < 0 || (n > 0 && (!type || !src || !dst))) {
    set_error("sp_degree_dynamic: invalid argument");
    return SP_ERR_INVALID;
  }
  if (n > 0) SP_TRY(update_graph(g, n, type, src, dst, weight));
  return sp_degree_centrality(g, deg);
}

extern "C" int sp_closeness(sp_graph_h g, const int32_t* weight, const int32_t* sources, int32_t nsrc, float* CC) {
  using namespace sp;
  if (!g || !sources || nsrc <= 0 || !CC) {
    set_error("sp_closeness: invalid argument");
    return SP_ERR_INVALID;
  }
  std::vector<int32_t> hs;
  SP_TRY(read_sources(g, sources, nsrc, hs, "sp_closeness"));
  cudaStream_t s = g->stream;
  dbuf<unsigned long long> sums;
  SP_TRY(sums.alloc(nsrc));
  SP_CHECK_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(unsigned long long) * nsrc, s));
  // every source's delta-stepping solve in batched cooperative launches (one CTA group
  // per source), the rows summed on the device
  SP_TRY(sssp_batch_sums(g, weight, hs, cen::sum_finite_rows, sums.p));
  std::vector<long long> hsum(nsrc);
  SP_TRY(copy_out(hsum.data(), sums.p, sizeof(long long) * nsrc, s));
  return write_closeness(g, hs, hsum, CC);
}

extern "C" int sp_closeness_unweighted(sp_graph_h g, const int32_t* sources, int32_t nsrc, float* CC) {
  using namespace sp;
  if (!g || !sources || nsrc <= 0 || !CC) {
    set_error("sp_closeness_unweighted: invalid argument");
    return SP_ERR_INVALID;
  }
  std::vector<int32_t> hs;
  SP_TRY(read_sources(g, sources, nsrc, hs, "sp_closeness_unweighted"));
  cudaStream_t s = g->stream;
  const int B = std::min(nsrc, 64);
  const size_t n = (size_t)B * g->V;
  dbuf<int32_t> lvl, srcs;
  dbuf<double> sig;
  dbuf<unsigned long long> sums;
  SP_TRY(lvl.alloc(n));
  SP_TRY(sig.alloc(n));
  SP_TRY(srcs.alloc(nsrc));
  SP_TRY(sums.alloc(nsrc));
  SP_CHECK_CUDA(cudaMemcpyAsync(srcs.p, hs.data(), sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
  SP_CHECK_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(unsigned long long) * nsrc, s));
  for (int k0 = 0; k0 < nsrc; k0 += B) {
    const int b = std::min(B, nsrc - k0);
    SP_TRY(bc_levels(g, srcs.p + k0, b, lvl.p, sig.p));
    cen::k_sum_except<<<num_sms() * 4, 256, 0, s>>>(lvl.p, g->V, b, -1, sums.p + k0);
    SP_CHECK_LAUNCH();
  }
  std::vector<long long> hsum(nsrc);
  SP_TRY(copy_out(hsum.data(), sums.p, sizeof(long long) * nsrc, s));
  return write_closeness(g, hs, hsum, CC);
}
