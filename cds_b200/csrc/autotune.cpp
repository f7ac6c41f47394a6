// autotune.cpp -- picks listing, peel and push-relabel launch shapes per
// clique size by timing candidates on sample graphs (cds_autotune in cds.h).
//
// The reference fixes its launch geometry at compile time (BLK_NUMS 216,
// BLK_DIM 1024, cudaCode/inc/common.h:30-36).  Here every candidate is timed
// with device events on the caller's graphs; the fastest per stage is kept in
// the context and, if a cache path is given, written as "k key value" lines
// that later calls read back instead of timing again.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "pipeline.h"

namespace {

bool load_cache(cds_ctx *c, uint32_t k, const char *path) {
  if (!path) return false;
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  bool any = false;
  cds::Tuning t = c->tune[k];
  while (std::getline(f, line)) {
    std::istringstream is(line);
    uint32_t kk;
    std::string key;
    int val;
    if (!(is >> kk >> key >> val) || kk != k) continue;
    // block sizes: whole warps within the ranges the kernels are built for
    const bool warps = val % 32 == 0;
    if (key == "list_warp_block" && warps && val >= 64 && val <= 512) t.list_warp_block = val;
    else if (key == "list_team_block" && warps && val >= 64 && val <= 512) t.list_team_block = val;
    else if (key == "flow_block" && warps && val >= 128 && val <= 512) t.flow_block = val;
    else if (key == "flow_rounds" && val >= 1 && val <= 1024) t.flow_rounds = val;
    else if (key == "list_warp_dmax" && val >= 32 && val <= 128) t.list_warp_dmax = val;
    else if (key == "peel_chunk" && val >= 32) t.peel_chunk = val;
    else if (key == "flow_warm" && val >= -1 && val <= 255) t.flow_warm = val;
    else if (key == "flow_inc_per_block" && val >= 0) t.flow_inc_per_block = val;
    else if (key == "peel_order" && (val == 0 || val == 1)) t.peel_order = val;
    else if (key == "peel_static" && val >= 0 && val <= 100) t.peel_static = val;
    else continue;
    any = true;
  }
  if (any) c->tune[k] = t;
  return any;
}

void save_cache(const cds_ctx *c, uint32_t k, const char *path) {
  if (!path) return;
  // keep the lines of other k values
  std::vector<std::string> keep;
  {
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
      std::istringstream is(line);
      uint32_t kk;
      if ((is >> kk) && kk != k) keep.push_back(line);
    }
  }
  std::ofstream f(path, std::ios::trunc);
  for (auto &l : keep) f << l << "\n";
  const cds::Tuning &t = c->tune[k];
  f << k << " list_warp_block " << t.list_warp_block << "\n";
  f << k << " list_team_block " << t.list_team_block << "\n";
  f << k << " flow_block " << t.flow_block << "\n";
  f << k << " flow_rounds " << t.flow_rounds << "\n";
  f << k << " list_warp_dmax " << t.list_warp_dmax << "\n";
  f << k << " peel_chunk " << t.peel_chunk << "\n";
  f << k << " flow_warm " << t.flow_warm << "\n";
  f << k << " flow_inc_per_block " << t.flow_inc_per_block << "\n";
  f << k << " peel_order " << t.peel_order << "\n";
  f << k << " peel_static " << t.peel_static << "\n";
}

// device time of one solve of every sample graph with the context's tuning
double time_solves(cds_ctx *c, cds_graph *const *graphs, size_t n, uint32_t k) {
  double ms = 0;
  for (size_t i = 0; i < n; i++) {
    cds::UnionGraph u;
    cds::build_union(c, c->stream, {graphs[i]}, u);
    cds_params p{};
    p.k = k;
    p.early_stop = -1;
    std::vector<cds::ProblemResult> res;
    cds::run_problem(c, c->stream, u, p, res);
    ms += res[0].t_ms[CDS_T_LIST] + res[0].t_ms[CDS_T_PEEL] + res[0].t_ms[CDS_T_EXACT];
  }
  return ms;
}

}  // namespace

extern "C" cds_status cds_autotune(cds_ctx *c, cds_graph *const *graphs, size_t n, uint32_t k,
                                   const char *cache_path) {
  if (!c || (n && !graphs) || k < 2 || k > CDS_MAX_K) return CDS_ERR_INPUT;
  if (load_cache(c, k, cache_path)) return CDS_OK;
  try {
    for (size_t i = 0; i < n; i++)
      if (!graphs[i] || graphs[i]->ctx != c) cds::fail(CDS_ERR_INPUT, "graph of another context");
    if (n == 0) return CDS_OK;
    time_solves(c, graphs, n, k);  // warm-up: pool allocations, module load
    struct Cand {
      int *field;
      std::vector<int> values;
    };
    cds::Tuning &t = c->tune[k];
    std::vector<Cand> cands = {
        {&t.list_warp_block, {128, 256, 512}},
        {&t.list_warp_dmax, {32, 64, 128}},
        {&t.list_team_block, {256, 512}},
        {&t.flow_rounds, {4, 8, 16, 32}},
        {&t.flow_block, {256, 512}},
        {&t.peel_chunk, {256, 512, 1024}},
        {&t.flow_warm, {-1, 0, 1, 3, 6}},
        {&t.flow_inc_per_block, {0, 4096, 16384, 65536}},
        {&t.peel_order, {0, 1}},
        {&t.peel_static, {100, 75, 50}},
    };
    // coordinate descent: one field at a time, the others at their best
    for (auto &cd : cands) {
      int best = *cd.field;
      double best_ms = 1e300;
      for (int v : cd.values) {
        *cd.field = v;
        const double ms = time_solves(c, graphs, n, k);
        if (ms < best_ms) {
          best_ms = ms;
          best = v;
        }
      }
      *cd.field = best;
    }
    save_cache(c, k, cache_path);
  } catch (const cds::Error &e) {
    std::lock_guard<std::mutex> g(c->mu);
    c->err = e.msg;
    return e.status;
  }
  return CDS_OK;
}
