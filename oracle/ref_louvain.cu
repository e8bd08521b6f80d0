// ORACLE — test infrastructure only. Compiled from the reference's own
// graphcode/dynamic_louvain_community_detection/communitydetection_sequential_allocation.cu
// (included in place, its main renamed) into oracle/_ref/ref_louvain;
// tests/golden/make_gpu_fixtures.py runs it on one GPU and commits the modularity of
// its partitions as golden fixtures. Nothing in the product links it.
//
//   ref_louvain <graph.txt> <communities.bin>
//
// runs the static half of the reference's main (:1431-1485): parseGraph on a
// "p q w" edge list (both directions of every undirected edge), m from
// computeGraphWeight, the vertex-community map set to the identity, then louvain()
// (local moves by moveNodes until Q stops rising by 1e-8, aggregation, repeated while
// any community merged). The dynamic half (new-edge batches) is not run. The final
// community of every vertex 0 .. num_nodes-1 is written as int32 (num_nodes = the
// largest id in the file + 1), followed by nothing else.
#define main louvain_reference_main
#include "dynamic_louvain_community_detection/communitydetection_sequential_allocation.cu"
#undef main

#include <cstdio>

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <graph.txt> <communities.bin>\n", argv[0]);
    return 1;
  }
  Graph G;
  parseGraph(argv[1], G);
  G.d_m = computeGraphWeight(G);
  VertexCommunityMap vertex_community_map;
  vertex_community_map.size = G.num_nodes;
  cudaMallocManaged(&vertex_community_map.d_vertex_map, vertex_community_map.size * sizeof(int));
  const int threadsPerBlock = 1024;
  const int blocksPerGrid = (G.num_nodes + threadsPerBlock - 1) / threadsPerBlock;
  initializeVertexCommunityMap<<<blocksPerGrid, threadsPerBlock>>>(vertex_community_map.d_vertex_map, G.num_nodes);
  cudaDeviceSynchronize();
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start);
  louvain(G, vertex_community_map);
  cudaEventRecord(stop);
  cudaEventSynchronize(stop);
  float ms = 0;
  cudaEventElapsedTime(&ms, start, stop);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    fprintf(stderr, "ref_louvain: %s\n", cudaGetErrorString(err));
    return 2;
  }
  FILE* o = fopen(argv[2], "wb");
  if (!o) return 3;
  fwrite(vertex_community_map.d_vertex_map, sizeof(int), vertex_community_map.size, o);
  fclose(o);
  printf("louvain_ms %.3f nodes %d\n", ms, vertex_community_map.size);
  return 0;
}
