// main.cpp -- command-line driver with the reference's surface:
//
//   main <graph> <k> <pSize> <cpSize> <glBufferSize> <partitionSize> <earlyStop>
//        [--search dinkelbach|bisect|core] [--device N]
//
// Arguments and stdout keys follow cudaCode/main.cu:865-1107, including the
// per-component lb= / ub= / eub= lines (eub, the reference's entropy bound,
// is not computed: n/a); the answer lines (K:, Density:, Size:, densest
// subgraph:) follow the CPU program, cpuCode/c++/src/helpers.cpp:1580-1588,
// and Density_fraction: gives the exact value.  An approximate answer
// (earlyStop >= 0 that cut a flow short, or --search core: the densest core
// alone) adds Approximate:, Density_upper_bound: and Density_gap: lines.
// Exit status 0 on success, 1 on bad arguments (as the reference), 2 on a
// failed solve.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cds.h"

int main(int argc, const char *argv[]) {
  int nargs = argc;
  const char *search = "dinkelbach";
  int device = 0;
  for (int i = 8; i + 1 < argc; i += 2) {
    if (!std::strcmp(argv[i], "--search")) search = argv[i + 1];
    else if (!std::strcmp(argv[i], "--device")) device = std::atoi(argv[i + 1]);
    else {
      nargs = -1;
      break;
    }
  }
  if (nargs != 8 && !(argc > 8 && (argc - 8) % 2 == 0 && nargs != -1)) {
    std::printf("Server wrong input parameters!\n");
    return 1;
  }
  cds_params p{};
  p.k = (uint32_t)std::atoi(argv[2]);
  p.p_size = (uint32_t)std::atoi(argv[3]);
  p.cp_size = (uint32_t)std::atoi(argv[4]);
  p.gl_buffer_size = (uint32_t)std::atoi(argv[5]);
  p.partition_size = (uint32_t)std::atoi(argv[6]);
  p.early_stop = std::atoi(argv[7]);
  if (!std::strcmp(search, "bisect")) p.search = CDS_SEARCH_BISECT;
  else if (!std::strcmp(search, "core")) p.search = CDS_SEARCH_CORE;
  else if (!std::strcmp(search, "dinkelbach")) p.search = CDS_SEARCH_DINKELBACH;
  else {
    std::printf("Server wrong input parameters!\n");
    return 1;
  }

  cds_config cfg{};
  cfg.device = device;
  cds_ctx *ctx = nullptr;
  cds_status st = cds_create(&cfg, &ctx);
  if (st != CDS_OK) {
    std::fprintf(stderr, "cds_create: %s\n", cds_status_string(st));
    return 2;
  }
  cds_graph *g = nullptr;
  st = cds_graph_load_file(ctx, argv[1], &g);
  if (st != CDS_OK) {
    std::printf("Graph file Open Failed \n");
    std::fprintf(stderr, "%s\n", cds_last_error(ctx));
    cds_destroy(ctx);
    return 2;
  }
  uint32_t n = 0, maxd = 0;
  uint64_t m = 0;
  cds_graph_info(g, &n, &m, &maxd);
  std::printf("n=%u, m=%llu\n", n, (unsigned long long)m);
  std::printf("Max Degree=%u\n", maxd);

  cds_result r;
  st = cds_solve(ctx, g, &p, &r);
  if (st != CDS_OK) {
    std::fprintf(stderr, "cds_solve: %s: %s\n", cds_status_string(st), cds_last_error(ctx));
    cds_graph_free(g);
    cds_destroy(ctx);
    return 2;
  }
  if (r.total_cliques == 0) {
    std::printf("Max Density 0 Size 0\n");
    std::printf("Time taken: %.3f ms\n", r.t_ms[CDS_T_TOTAL]);
  } else {
    const double dens = r.den ? (double)r.num / (double)r.den : 0.0;
    const double core = r.core_den ? (double)r.core_num / (double)r.core_den : 0.0;
    std::printf("Final Max Density %.6g\n", dens);
    std::printf("Total Cliques=%llu\n", (unsigned long long)r.total_cliques);
    std::printf("Densest Core Density=%.6g\n", core);
    std::printf("Total Components=%u\n", r.n_components);
    std::printf("\n");
    std::printf("DAG Time =%.3f ms\n", r.t_ms[CDS_T_DAG]);
    std::printf("Clique Listing Time =%.3f ms\n", r.t_ms[CDS_T_LIST]);
    std::printf("Core Decompose Time =%.3f ms\n", r.t_ms[CDS_T_PEEL]);
    std::printf("Densest Core Time =%.3f ms\n", r.t_ms[CDS_T_CORE]);
    std::printf("Prune Time =%.3f ms\n", r.t_ms[CDS_T_PRUNE]);
    std::printf("Connected Component Time =%.3f ms\n", r.t_ms[CDS_T_COMPONENTS]);
    std::printf("Exact Time =%.3f ms\n", r.t_ms[CDS_T_EXACT]);
    std::printf("Time taken=%.3f ms\n", r.t_ms[CDS_T_TOTAL]);
    std::printf("\nMac Clique Core=%llu\n", (unsigned long long)r.max_core);
    std::printf("lb=");
    for (uint32_t i = 0; i < r.n_bounds; i++) std::printf("%g ", r.bound_lb[i]);
    std::printf("\nub=");
    for (uint32_t i = 0; i < r.n_bounds; i++) std::printf("%g ", r.bound_ub[i]);
    std::printf("\neub=n/a\n");
    std::printf("Densest_core_threshold=%llu\n", (unsigned long long)r.core_threshold);
    std::printf("Densest_core_size=%llu\n", (unsigned long long)r.core_size);
    std::printf("Remaining_edges_after_prune=%llu\n", (unsigned long long)r.pruned_edges);
    std::printf("Max_flow_solves=%u\n", r.flows);
    if (r.early_stopped) std::printf("Early_stopped=1\n");
    const bool approx = r.early_stopped || p.search == CDS_SEARCH_CORE;
    if (approx) {
      const double ub = r.ub_den ? (double)r.ub_num / (double)r.ub_den : 0.0;
      std::printf("Approximate: %s\n", p.search == CDS_SEARCH_CORE ? "densest core" : "early stop");
      std::printf("Density_upper_bound: %llu/%llu\n", (unsigned long long)r.ub_num,
                  (unsigned long long)r.ub_den);
      std::printf("Density_gap: %.6g\n", ub - dens);
    }
  }
  std::printf("K: %u\n", p.k);
  std::printf("Density: %.6g\n", r.den ? (double)r.num / (double)r.den : 0.0);
  std::printf("Density_fraction: %llu/%llu\n", (unsigned long long)r.num,
              (unsigned long long)r.den);
  std::printf("Size: %llu\n", (unsigned long long)r.size);
  std::printf("densest subgraph: ");
  for (uint64_t i = 0; i < r.size; i++) std::printf("%u ", r.vertices[i]);
  std::printf("\n");
  cds_result_free(&r);
  cds_graph_free(g);
  cds_destroy(ctx);
  return 0;
}
