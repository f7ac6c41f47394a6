// ref_dump: runs the reference CPU pipeline stage by stage through its public
// CDS methods and prints every intermediate result as one JSON object.
//
// Test infrastructure only.  This file holds no reference code: it includes
// the reference headers and is linked against the reference sources where they
// lie (see oracle/Makefile), and calls the public members declared in
// cpuCode/c++/inc/helpers.h:52-75, in the order CDS::DSD uses them
// (cpuCode/c++/src/helpers.cpp:1422-1537).
//
// usage: ref_dump <graph> <k> [ub1=1] [ub2=0] [stages=all|peel]
//
// The reference reads k from the first integer of a motif file
// (cpuCode/c++/src/graph.cpp:58-76) and uses nothing else of it, so the Motif
// object is filled in directly.
#include "inc/common.h"
#include "inc/graph.h"
#include "inc/helpers.h"

#include <cstdio>

static void put_d(double x) { std::printf("%.17g", x); }

int main(int argc, const char *argv[]) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_dump <graph> <k> [ub1] [ub2] [all|peel]\n");
    return 2;
  }
  std::string path = argv[1];
  unsigned k = (unsigned)std::atoi(argv[2]);
  bool ub1 = argc > 3 ? std::atoi(argv[3]) != 0 : true;
  bool ub2 = argc > 4 ? std::atoi(argv[4]) != 0 : false;
  bool all = !(argc > 5 && std::string(argv[5]) == "peel");

  Graph graph(path);
  Motif motif;
  motif.size = k;
  motif.type = 1;
  motif.count = 1;
  CDS cds(&graph, &motif, ub1, ub2);

  std::vector<std::vector<double>> results;
  cds.cliqueCoreDecompose(results);

  std::printf("{\"n\": %u, \"k\": %u, \"total_cliques\": %ld", graph.n, k,
              graph.totalCliques);
  std::printf(", \"clique_degree\": [");
  for (unsigned i = 0; i < graph.n; i++)
    std::printf("%s%ld", i ? ", " : "", graph.cliqueDegree[i]);
  std::printf("], \"peel\": [");
  for (size_t i = 0; i < results.size(); i++) {
    std::printf("%s[", i ? ", " : "");
    for (int j = 0; j < 4; j++) {
      if (j) std::printf(", ");
      put_d(results[i][j]);
    }
    std::printf("]");
  }
  std::printf("]");

  if (all) {
    DensestCoreData dc;
    cds.locateDensestCore(results, dc);
    std::printf(", \"densest_core\": {\"lower_bound\": %d, \"del_vertex_index\": %d, "
                "\"density\": ",
                dc.lowerBound, dc.delVertexIndex);
    put_d(dc.density);
    std::printf(", \"max_clique_core\": %d, \"vertices\": [", dc.maxCliqueCore);
    for (size_t i = 0; i < dc.reverseMap.size(); i++)
      std::printf("%s%u", i ? ", " : "", dc.reverseMap[i]);
    size_t core_arcs = 0;
    for (auto &row : dc.graph) core_arcs += row.size();
    std::printf("], \"edges\": %zu}", core_arcs / 2);

    std::unordered_map<std::string, std::vector<int>> cliqueData;
    std::vector<long> cliqueDegree;
    cds.cliqueEnumerationListRecord(dc.graph, cliqueData, cliqueDegree, k);
    std::printf(", \"core_cliques\": %zu", cliqueData.size());

    std::vector<std::vector<ui>> pruned;
    int valid = cds.pruneInvalidEdges(dc.graph, pruned, cliqueData);
    std::printf(", \"pruned_edges\": %d", valid);

    std::vector<ConnectedComponentData> comps;
    cds.connectedComponentDecompose(pruned, cliqueData, comps);
    std::printf(", \"components\": [");
    for (size_t i = 0; i < comps.size(); i++) {
      std::printf("%s{\"size\": %d, \"cliques\": %ld, \"first\": %u}", i ? ", " : "",
                  comps[i].size, comps[i].totalCliques,
                  dc.reverseMap[comps[i].reverseMap.empty() ? 0 : comps[i].reverseMap[0]]);
    }
    std::printf("]");

    finalResult fr;
    float u1 = 0.0f, u2 = 0.0f;
    cds.dynamicExact(comps, dc, fr, u1, u2, ub1, ub2);
    std::printf(", \"result\": {\"density\": ");
    put_d(fr.density);
    std::printf(", \"size\": %u, \"vertices\": [", fr.size);
    for (size_t i = 0; i < fr.verticies.size(); i++)
      std::printf("%s%u", i ? ", " : "", fr.verticies[i]);
    std::printf("]}");
  }
  std::printf("}\n");
  return 0;
}
