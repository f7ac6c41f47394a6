// pipeline.h -- problem-level orchestration shared by the C ABI entry points.
#pragma once
#include "stages.h"

namespace cds {

// Device-time marks on a stream, read once at the end (no host wait per
// stage): mark() records an event and returns its index; ms(a, b) is the time
// between two marks once the stream has passed the last one.
struct StageClock {
  std::vector<cudaEvent_t> ev;
  cudaStream_t s;
  explicit StageClock(cudaStream_t s_) : s(s_) {}
  int mark();
  double ms(int a, int b);  // after the last mark completed
  void wait();              // waits for the last mark
  ~StageClock();
};

// A graph or a disjoint union of graphs (instance i owns a vertex range).
struct UnionGraph {
  uint32_t n = 0;
  uint64_t nnz = 0;
  const uint64_t *off = nullptr;
  const uint32_t *adj = nullptr;
  DBuf<uint64_t> own_off;
  DBuf<uint32_t> own_adj;
  Instances inst;
};
void build_union(cds_ctx *c, cudaStream_t s, const std::vector<const cds_graph *> &gs,
                 UnionGraph &u);

struct ProblemResult {
  uint64_t num = 0, den = 0;
  uint64_t total_cliques = 0, max_core = 0, core_threshold = 0;
  uint64_t core_num = 0, core_den = 0, core_size = 0, core_cliques = 0, pruned_edges = 0;
  uint32_t n_components = 0, flows = 0, early_stopped = 0, levels = 0;
  uint64_t ub_num = 0, ub_den = 1;     // proven upper bound of the optimum density
  std::vector<double> bound_lb, bound_ub;  // per component with cliques (lb=, ub= lines)
  double t_ms[CDS_T_COUNT] = {0};
  std::vector<uint32_t> vertices;
};

void run_problem(cds_ctx *c, cudaStream_t s, UnionGraph &u, const cds_params &prm,
                 std::vector<ProblemResult> &res, const CountHook *on_count = nullptr);

// Pinned host memory for one bulk transfer, freed at scope exit.
struct PinnedHost {
  char *p = nullptr;
  explicit PinnedHost(size_t bytes);
  ~PinnedHost();
  PinnedHost(const PinnedHost &) = delete;
  PinnedHost &operator=(const PinnedHost &) = delete;
};

// Adjacency-list text already in device memory -> a canonical CSR graph
// (parse.cu).  CDS_ERR_INPUT on malformed text.
void parse_adjlist_device(cds_ctx *c, cudaStream_t s, const uint8_t *txt, uint64_t len, cds_graph **out);

// result conversion and graph upload shared by the batch and server paths
void fill_result(const ProblemResult &r, cds_result *out);
cds_status graph_upload(cds_ctx *c, cudaStream_t s, const uint64_t *off, const uint32_t *adj,
                        uint32_t n, cds_graph **out);

}  // namespace cds
