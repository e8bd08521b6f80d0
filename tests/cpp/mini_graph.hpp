// Test stand-in for the reference's `graph` class (graphcode/graph.hpp:31-57):
// only the public members the generated entry points and starplat_b200.hpp use.
#pragma once
#include <cstdint>
#include <cstdio>
#include <vector>

class graph {
 public:
  int32_t* indexofNodes = nullptr;
  int32_t* edgeList = nullptr;
  int32_t* rev_indexofNodes = nullptr;
  int32_t* srcList = nullptr;
  int num_nodes() { return V; }
  int num_edges() { return E; }
  int32_t* getEdgeLen() { return edgeLen; }

  // binary CSR written by the test: V, E, indexofNodes, edgeList, edgeLen, rev_indexofNodes, srcList
  bool load(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    bool ok = std::fread(&V, 4, 1, f) == 1 && std::fread(&E, 4, 1, f) == 1;
    off_.resize(V + 1), adj_.resize(E), w_.resize(E), roff_.resize(V + 1), radj_.resize(E);
    ok = ok && std::fread(off_.data(), 4, V + 1, f) == (size_t)V + 1 && std::fread(adj_.data(), 4, E, f) == (size_t)E &&
         std::fread(w_.data(), 4, E, f) == (size_t)E && std::fread(roff_.data(), 4, V + 1, f) == (size_t)V + 1 &&
         std::fread(radj_.data(), 4, E, f) == (size_t)E;
    std::fclose(f);
    indexofNodes = off_.data(), edgeList = adj_.data(), edgeLen = w_.data();
    rev_indexofNodes = roff_.data(), srcList = radj_.data();
    return ok;
  }

 private:
  int V = 0, E = 0;
  int32_t* edgeLen = nullptr;
  std::vector<int32_t> off_, adj_, w_, roff_, radj_;
};
