// ORACLE — test infrastructure only. Compiled from the reference's own
// graphcode/manual_cuda/bcManualv5.cu (included in place, its main renamed) into
// oracle/_ref/ref_bc_manual; tests/golden/make_gpu_fixtures.py runs it on one GPU
// and commits its outputs as golden fixtures. Nothing in the product links it.
//
// Two modes:
//   ref_bc_manual main <graph.txt> <sources.txt>
//       the reference's own main (bcManualv5.cu:289-336): graph::parseGraph, then
//       BC(G, sources, printAns=true), which prints "i BC[i]" for i = 0..8;
//   ref_bc_manual csr <graph.bin> <out.bin>
//       the reference kernels (initialize, bc_forward_pass, incHop, bc_backward_pass,
//       accumulate_bc) launched in the order BC() launches them
//       (bcManualv5.cu:198-253), over a CSR given in binary, so that graphs too large
//       for parseGraph can be used and the whole BC vector is written out.
//       graph.bin: int32 V, int64 E, int32 off[V+1], int32 adj[E], int32 n,
//       int32 sources[n] (BC() walks a std::set, so sources ascending, distinct);
//       out.bin: double BC[V] (the reference halves each dependency: BC += delta / 2).
#define main bc_manual_reference_main
#include "manual_cuda/bcManualv5.cu"
#undef main

#include <cstdint>
#include <cstdio>
#include <vector>

namespace {

bool read_all(FILE* f, void* p, size_t bytes) { return fread(p, 1, bytes, f) == bytes; }

int run_csr(const char* in_path, const char* out_path) {
  FILE* f = fopen(in_path, "rb");
  if (!f) return 2;
  int32_t V = 0;
  int64_t E = 0;
  if (!read_all(f, &V, 4) || !read_all(f, &E, 8) || V <= 0 || E < 0) return 3;
  std::vector<int32_t> off(V + 1), adj(E > 0 ? E : 1);
  int32_t n = 0;
  if (!read_all(f, off.data(), 4 * (size_t)(V + 1)) || !read_all(f, adj.data(), 4 * (size_t)E) ||
      !read_all(f, &n, 4) || n < 0)
    return 4;
  std::vector<int32_t> src(n > 0 ? n : 1);
  if (!read_all(f, src.data(), 4 * (size_t)n)) return 5;
  fclose(f);
  // the checks graph::parseGraph's CSR satisfies, so the kernels stay inside the arrays
  if (off[0] != 0 || off[V] != E) return 6;
  for (int32_t v = 0; v < V; ++v)
    if (off[v + 1] < off[v]) return 6;
  for (int64_t e = 0; e < E; ++e)
    if (adj[e] < 0 || adj[e] >= V) return 6;
  for (int32_t i = 0; i < n; ++i)
    if (src[i] < 0 || src[i] >= V || (i > 0 && src[i] <= src[i - 1])) return 7;

  int *d_offset, *d_edgeList, *d_edgeLen, *d_level, *d_hops_from_source;
  double *d_sigma, *d_delta, *d_nodeBC;
  bool* d_finished;
  cudaMalloc(&d_offset, sizeof(int) * (V + 1));
  cudaMalloc(&d_edgeList, sizeof(int) * (E > 0 ? E : 1));
  cudaMalloc(&d_edgeLen, sizeof(int) * (E > 0 ? E : 1));  // unused by the kernels, passed as BC() does
  cudaMemcpy(d_offset, off.data(), sizeof(int) * (V + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_edgeList, adj.data(), sizeof(int) * E, cudaMemcpyHostToDevice);
  cudaMemset(d_edgeLen, 0, sizeof(int) * (E > 0 ? E : 1));
  cudaMalloc(&d_sigma, sizeof(double) * V);
  cudaMalloc(&d_delta, sizeof(double) * V);
  cudaMalloc(&d_nodeBC, sizeof(double) * V);
  cudaMemset(d_nodeBC, 0, sizeof(double) * V);  // BC() leaves it as cudaMalloc returns it
  cudaMalloc(&d_finished, sizeof(bool));
  cudaMalloc(&d_hops_from_source, sizeof(int));
  cudaMalloc(&d_level, sizeof(int) * V);

  // launch shape of BC() (bcManualv5.cu:198-203)
  unsigned block_size = V, num_blocks = 1;
  if (V > 1024) {
    block_size = 1024;
    num_blocks = (V + block_size - 1) / block_size;
  }
  for (int32_t k = 0; k < n; ++k) {
    const unsigned s = (unsigned)src[k];
    int hops_from_source = 0;
    bool finished = false;
    initialize<<<num_blocks, block_size>>>(d_sigma, d_delta, d_level, d_hops_from_source, s, V);
    do {  // forward pass, one level per launch (bcManualv5.cu:213-230)
      finished = true;
      cudaMemcpy(d_finished, &finished, sizeof(bool), cudaMemcpyHostToDevice);
      bc_forward_pass<<<num_blocks, block_size>>>(d_offset, d_edgeList, d_edgeLen, d_sigma, d_level,
                                                  d_hops_from_source, V, d_finished);
      cudaDeviceSynchronize();
      ++hops_from_source;
      incHop<<<1, 1>>>(d_hops_from_source);
      cudaDeviceSynchronize();
      cudaMemcpy(&finished, d_finished, sizeof(bool), cudaMemcpyDeviceToHost);
    } while (!finished);
    hops_from_source--;  // backward pass (bcManualv5.cu:242-250)
    cudaMemcpy(d_hops_from_source, &hops_from_source, sizeof(int), cudaMemcpyHostToDevice);
    while (hops_from_source > 1) {
      bc_backward_pass<<<num_blocks, block_size>>>(d_offset, d_edgeList, d_edgeLen, d_sigma, d_delta, d_nodeBC,
                                                   d_level, d_hops_from_source, V);
      --hops_from_source;
      cudaMemcpy(d_hops_from_source, &hops_from_source, sizeof(int), cudaMemcpyHostToDevice);
    }
    accumulate_bc<<<num_blocks, block_size>>>(d_delta, d_nodeBC, d_level, s, V);
    cudaDeviceSynchronize();
  }
  std::vector<double> bc(V);
  cudaMemcpy(bc.data(), d_nodeBC, sizeof(double) * V, cudaMemcpyDeviceToHost);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    fprintf(stderr, "ref_bc_manual: %s\n", cudaGetErrorString(err));
    return 8;
  }
  FILE* o = fopen(out_path, "wb");
  if (!o) return 9;
  fwrite(bc.data(), sizeof(double), V, o);
  fclose(o);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 4 && std::string(argv[1]) == "main") {
    char p[] = "-p";
    char* args[] = {argv[0], argv[2], argv[3], p, nullptr};
    return bc_manual_reference_main(4, args);
  }
  if (argc == 4 && std::string(argv[1]) == "csr") {
    const int rc = run_csr(argv[2], argv[3]);
    if (rc) fprintf(stderr, "ref_bc_manual csr: failed (%d)\n", rc);
    return rc;
  }
  fprintf(stderr, "usage: %s main <graph.txt> <sources.txt> | csr <graph.bin> <out.bin>\n", argv[0]);
  return 1;
}
