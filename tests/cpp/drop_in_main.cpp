// Driver in the shape of the reference's main_functions/*main.cpp: builds a graph,
// calls the generated entry points (now from starplat_b200.hpp) and prints results.
#include <cstdio>
#include <set>
#include <vector>

#ifdef GRAPH_HEADER
#include GRAPH_HEADER
#endif
#include "starplat_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
#if defined(LIBRARY_PARSE)  // the library reads the text file (starplat_b200::Graph)
  starplat_b200::Graph g(argv[1]);
  g.parseGraph();
#elif defined(PARSE_TEXT)  // the reference's graph::parseGraph
  graph g(argv[1]);
  g.parseGraph();
#else
  graph g;
  if (!g.load(argv[1])) return 3;
#endif
  const int V = g.num_nodes();
  std::printf("V %d E %d\n", V, g.num_edges());
  long tc = Compute_TC(g);
  std::printf("TC %ld\n", tc);
  std::vector<float> pr(V);
  ComputePageRank(g, 1e-6f, 0.85f, 100, pr.data());
  std::printf("PR");
  for (int v = 0; v < V; ++v) std::printf(" %.9g", pr[v]);
  std::printf("\n");
  std::vector<int> dist(V), w(g.getEdgeLen(), g.getEdgeLen() + g.num_edges());
  Compute_SSSP(g, dist.data(), w.data(), atoi(argv[2]));
  std::printf("SSSP");
  for (int v = 0; v < V; ++v) std::printf(" %d", dist[v]);
  std::printf("\n");
  std::set<int> sources;
  for (int v = 0; v < V; v += 3) sources.insert(v);
  std::vector<float> bc(V);
  Compute_BC(g, bc.data(), sources);
  std::printf("BC");
  for (int v = 0; v < V; ++v) std::printf(" %.9g", bc[v]);
  std::printf("\n");
  std::printf("CD %.12f\n", Compute_CD(g, nullptr));
  std::vector<int> cf(V), deg(V);
  staticClusteringCoeff(g, cf.data());
  std::printf("LCC");
  for (int v = 0; v < V; ++v) std::printf(" %d", cf[v]);
  std::printf("\n");
  Degree(g, deg.data());
  std::printf("DEG");
  for (int v = 0; v < V; ++v) std::printf(" %d", deg[v]);
  std::printf("\n");
  std::vector<float> cc(V), ccu(V);
  Compute_CC(g, cc.data(), sources);
  std::printf("CC");
  for (int v = 0; v < V; ++v) std::printf(" %.9g", cc[v]);
  std::printf("\n");
  Compute_CC_Unweighted(g, ccu.data(), sources);
  std::printf("CCU");
  for (int v = 0; v < V; ++v) std::printf(" %.9g", ccu[v]);
  std::printf("\n");
  // a batch of updates shaped like the reference's update records: drop the first
  // edge of vertex 1 (both directions) and add 0 <-> V-1
  struct Upd {
    char type;
    int source, destination, weight;
  };
  std::vector<Upd> batch;
  const int* off = g.indexofNodes;
  const int* adj = g.edgeList;
  if (off[2] > off[1]) {
    batch.push_back({'d', 1, adj[off[1]], 0});
    batch.push_back({'d', adj[off[1]], 1, 0});
  }
  batch.push_back({'a', 0, V - 1, 3});
  batch.push_back({'a', V - 1, 0, 3});
  starplat_b200::apply_updates(g, batch, 0, (int)batch.size());
  std::printf("TCU %ld\n", Compute_TC(g));
  // DynTC's batch: drop 0 <-> V-1 again (incremental: the graph and batch are symmetric)
  std::vector<Upd> batch1 = {{'d', 0, V - 1, 0}, {'d', V - 1, 0, 0}};
  std::printf("TCD %ld\n", starplat_b200::dynamic_tc(g, batch1, 0, 2, Compute_TC(g)));
  // DynCF's batch (add 0 <-> V-1 back) from the counts of the current graph, then
  // DynDegree's (add 3 -> V-4)
  staticClusteringCoeff(g, cf.data());
  std::vector<Upd> batch_cf = {{'a', 0, V - 1, 1}, {'a', V - 1, 0, 1}};
  starplat_b200::dynamic_clustering_coeff(g, batch_cf, 0, 2, cf.data());
  std::printf("LCCU");
  for (int v = 0; v < V; ++v) std::printf(" %d", cf[v]);
  std::printf("\n");
  std::vector<Upd> batch_deg = {{'a', 3, V - 4, 1}};
  starplat_b200::dynamic_degree(g, batch_deg, 0, 1, deg.data());
  std::printf("DEGU");
  for (int v = 0; v < V; ++v) std::printf(" %d", deg[v]);
  std::printf("\n");
  // DynPR's batch on the updated copy: add 1 <-> V-2 and refresh the ranks from the
  // previous ones
  std::vector<Upd> batch2 = {{'a', 1, V - 2, 2}, {'a', V - 2, 1, 2}};
  starplat_b200::dynamic_pagerank(g, batch2, 0, 2, 1e-9f, 0.85f, 100, pr.data());
  std::printf("PRU");
  for (int v = 0; v < V; ++v) std::printf(" %.9g", pr[v]);
  std::printf("\n");
  // a batch with a deletion solves again (on the copy's edgeLen); additions only resume
  starplat_b200::dynamic_sssp(g, std::vector<Upd>{{'d', 0, 0, 0}}, 0, 1, dist.data(), atoi(argv[2]));
  std::vector<Upd> batch3 = {{'a', 2, V - 3, 1}, {'a', V - 3, 2, 1}};
  starplat_b200::dynamic_sssp(g, batch3, 0, 2, dist.data(), atoi(argv[2]));
  std::printf("SSSPU");
  for (int v = 0; v < V; ++v) std::printf(" %d", dist[v]);
  std::printf("\n");
  starplat_b200::invalidate(g);
  return 0;
}
