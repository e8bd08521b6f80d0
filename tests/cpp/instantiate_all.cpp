// Compile-only check: instantiates every template of starplat_b200.hpp (templates that no
// driver calls are otherwise never type-checked). Never run.
#include <set>
#include <vector>

#include "mini_graph.hpp"
#include "starplat_b200.hpp"

struct Upd {
  char type;
  int source, destination, weight;
};

void instantiate_all(graph& g, std::vector<Upd>& batch, std::set<int>& seeds, int* i, float* f) {
  (void)Compute_TC(g);
  ComputePageRank(g, 1e-6f, 0.85f, 100, f);
  Compute_PR(g, 1e-6f, 0.85f, 100, f);
  Compute_SSSP(g, i, i, 0);
  Compute_BC(g, f, seeds);
  (void)Compute_CD(g, i);
  staticClusteringCoeff(g, i);
  Degree(g, i);
  Compute_CC(g, f, seeds);
  Compute_CC_Unweighted(g, f, seeds);
  starplat_b200::apply_updates(g, batch, 0, 1);
  starplat_b200::dynamic_sssp(g, batch, 0, 1, i, 0);
  (void)starplat_b200::dynamic_tc(g, batch, 0, 1, 0L);
  starplat_b200::dynamic_clustering_coeff(g, batch, 0, 1, i);
  starplat_b200::dynamic_degree(g, batch, 0, 1, i);
  starplat_b200::dynamic_bc(g, batch, 0, 1, f, seeds);
  starplat_b200::dynamic_pagerank(g, batch, 0, 1, 1e-6f, 0.85f, 100, f);
  starplat_b200::invalidate(g);
}
