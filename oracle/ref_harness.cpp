// ORACLE (reference side) — test infrastructure only; never linked by the product.
//
// Compiled by oracle/Makefile directly against the reference's own CSR container
// (graphcode/graph.hpp, taken from where it lies in the reference checkout) into
// oracle/_ref/libspref.so. It exposes:
//   * ref_parse_graph: graph::parseGraph (graph.hpp:464-865) on a text edge list,
//     returning its CSR arrays — pins the CSR layout the kernels consume;
//   * ref_tc: the generated OpenMP triangle count loop calling the reference's
//     own graph::check_if_nbr / getNeighbors (graph.hpp:233-287, 982-1023) on a
//     graph object whose CSR fields are filled from given arrays;
//   * ref_lcc: the same loop with the clustering_coeff DSL body (one added to the
//     counts of all three vertices of each triangle found), sequential.
//
// Shim needed to compile graph.hpp without MKL: OMP_GNN.hpp is skipped
// (it includes <mkl.h>), the five GNN entry points graph.hpp:1244-1300 calls
// are declared, and `graph` is forward-declared because abstractGraph.hpp:30
// names it before its definition. Private members are opened so the harness can
// attach arrays it built itself (graph.hpp keeps edgeLen private).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <string.h>
#include <stdlib.h>
#include <unordered_set>
#include <vector>
#include <atomic>
#include <omp.h>

#define OMP_GNN_HPP 1
class graph;
void init_omp(std::vector<int> neuronsPerLayer, std::string initWeights, std::string folderPath);
void forward_omp(std::string modelType, std::string aggregationType);
void backprop_omp(std::string modelType, std::string aggregationType, int epoch);
double compute_accuracy_omp();
double compute_loss_omp();
#define private public
#include "graph.hpp"
#undef private

void init_omp(std::vector<int>, std::string, std::string) {}
void forward_omp(std::string, std::string) {}
void backprop_omp(std::string, std::string, int) {}
double compute_accuracy_omp() { return 0; }
double compute_loss_omp() { return 0; }

namespace {
struct parsed {
  graph* g;
};
}  // namespace

extern "C" {

// Parse a text edge list with graph::parseGraph. Returns a handle; sizes via
// ref_graph_sizes, arrays via ref_graph_copy. num_nodes() is max id + 1.
void* ref_parse_graph(const char* path) {
  graph* g = new graph(strdup(path));
  g->parseGraph();
  return g;
}

void ref_graph_sizes(void* h, int32_t* V, int32_t* E) {
  graph* g = (graph*)h;
  *V = g->num_nodes();
  *E = g->num_edges();
}

void ref_graph_copy(void* h, int32_t* off, int32_t* adj, int32_t* w, int32_t* roff,
                    int32_t* radj, int32_t* emap) {
  graph* g = (graph*)h;
  int32_t V = g->num_nodes(), E = g->num_edges();
  std::memcpy(off, g->indexofNodes, sizeof(int32_t) * (V + 1));
  std::memcpy(adj, g->edgeList, sizeof(int32_t) * E);
  std::memcpy(w, g->edgeLen, sizeof(int32_t) * E);
  std::memcpy(roff, g->rev_indexofNodes, sizeof(int32_t) * (V + 1));
  std::memcpy(radj, g->srcList, sizeof(int32_t) * E);
  std::memcpy(emap, g->edgeMap, sizeof(int32_t) * E);
}

void ref_graph_free(void* h) { (void)h; /* graph's destructor frees arrays it did not allocate here; leak intentionally */ }

// Generated OpenMP Compute_TC loop body with the reference's check_if_nbr.
// vstride > 1 samples every vstride-th outer vertex starting at vfirst.
int64_t ref_tc(int32_t V, const int32_t* off, const int32_t* adj, int nthreads, int32_t vfirst,
               int32_t vstride) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  if (vstride < 1) vstride = 1;
  graph g((char*)"");
  int32_t E = off[V];
  g.nodesTotal = V - 1;
  g.edgesTotal = E;
  g.indexofNodes = const_cast<int32_t*>(off);
  g.edgeList = const_cast<int32_t*>(adj);
  std::vector<int32_t> wts(E, 1);
  g.edgeLen = wts.data();
  g.srcList = nullptr;
  g.diff_edgeList = nullptr;
  int64_t triangle_count = 0;
#pragma omp parallel for reduction(+ : triangle_count) schedule(dynamic, 16)
  for (int32_t v = vfirst; v < V; v += vstride) {
    for (int32_t edge = g.indexofNodes[v]; edge < g.indexofNodes[v + 1]; edge++) {
      int32_t u = g.edgeList[edge];
      if (u < v) {
        for (int32_t edge2 = g.indexofNodes[v]; edge2 < g.indexofNodes[v + 1]; edge2++) {
          int32_t w = g.edgeList[edge2];
          if (w > v) {
            if (g.check_if_nbr(u, w)) triangle_count += 1;
          }
        }
      }
    }
  }
  // detach borrowed arrays so ~graph does not free them
  g.edgeLen = nullptr;
  g.edgeList = nullptr;
  g.srcList = nullptr;
  return triangle_count;
}

// Generated loop of staticClusteringCoeff (staticDSLCodes/clustering_coeff:1-14)
// with the reference's check_if_nbr; cf[V] is overwritten.
void ref_lcc(int32_t V, const int32_t* off, const int32_t* adj, int32_t* cf) {
  graph g((char*)"");
  int32_t E = off[V];
  g.nodesTotal = V - 1;
  g.edgesTotal = E;
  g.indexofNodes = const_cast<int32_t*>(off);
  g.edgeList = const_cast<int32_t*>(adj);
  std::vector<int32_t> wts(E, 1);
  g.edgeLen = wts.data();
  g.srcList = nullptr;
  g.diff_edgeList = nullptr;
  for (int32_t v = 0; v < V; v++) cf[v] = 0;
  for (int32_t v = 0; v < V; v++) {
    for (int32_t edge = g.indexofNodes[v]; edge < g.indexofNodes[v + 1]; edge++) {
      int32_t u = g.edgeList[edge];
      if (u < v) {
        for (int32_t edge2 = g.indexofNodes[v]; edge2 < g.indexofNodes[v + 1]; edge2++) {
          int32_t w = g.edgeList[edge2];
          if (w > v && g.check_if_nbr(u, w)) {
            cf[v] += 1;
            cf[u] += 1;
            cf[w] += 1;
          }
        }
      }
    }
  }
  // detach borrowed arrays so ~graph does not free them
  g.edgeLen = nullptr;
  g.edgeList = nullptr;
  g.srcList = nullptr;
}

}  // extern "C"
