// stages.h -- device-side data of one solve and the stage functions that
// produce it.  A "problem" is one graph or a disjoint union of instances
// (batched solves); every stage works on the union, and per-instance results
// come from the instance table.
#pragma once
#include <functional>

#include "cds_internal.h"

namespace cds {

struct Dag {
  uint32_t n = 0;
  uint32_t max_out = 0;
  DBuf<uint32_t> deg;     // [n] undirected degree
  DBuf<uint32_t> outdeg;  // [n] out-degree
  DBuf<uint64_t> off;     // [n+1] row starts (rows padded to 4 entries)
  DBuf<uint32_t> adj;     // out-neighbours, ascending id, 0xFFFFFFFF padding
};
void build_dag(cds_ctx *c, cudaStream_t s, const uint64_t *off, const uint32_t *adj,
               uint32_t n, Dag &dag);

struct Cliques {
  uint32_t k = 0;
  uint64_t count = 0;
  DBuf<unsigned long long> cdeg64;  // [n] clique degree of every vertex, exact
  DBuf<uint32_t> cdeg;     // [n] the same as u32 (materialised listings only; every
                           // clique degree below 2^32, else CDS_ERR_OVERFLOW)
  DBuf<uint64_t> base;     // [n+1] first clique rooted at each vertex
  DBuf<uint32_t> members;  // [count*k] clique records (k ids each)
};
// Called with |Psi| once the count pass is done, before anything sized by it
// is allocated (the server reserves device memory there; it may block).
using CountHook = std::function<void(uint64_t cliques)>;

// Counts (and, if materialize, writes) every k-clique.  The count and the
// u64 clique degrees have no 2^32 cap; a materialised listing also narrows
// the clique degrees to u32 for the later stages (CDS_ERR_OVERFLOW when one
// reaches 2^32).
void list_cliques(cds_ctx *c, cudaStream_t s, const Dag &dag, uint32_t k, bool materialize,
                  const Tuning &t, Cliques &out, const CountHook *on_count = nullptr);

// Instance table of a problem: instance i owns vertices [vbeg[i], vbeg[i+1]).
struct Instances {
  uint32_t count = 1;
  std::vector<uint32_t> h_vbeg;  // [count+1]
  DBuf<uint32_t> vbeg;           // [count+1]
  DBuf<uint32_t> of_vertex;      // [n] instance of each vertex (count > 1 only)
};

struct PeelOut {
  DBuf<uint32_t> core;              // [n] clique-core number
  DBuf<uint32_t> cmin;              // [m] smallest core number among each clique's members
  uint32_t max_core = 0;
  std::vector<uint64_t> best_num;   // per instance: best core density
  std::vector<uint64_t> best_den;
  std::vector<uint32_t> inst_max_core;
  std::vector<uint32_t> inst_levels;  // per instance: distinct core numbers
  std::vector<uint32_t> best_level;   // per instance: L of the densest core {core >= L}
  uint32_t levels = 0;                // the largest of inst_levels
};
void peel(cds_ctx *c, cudaStream_t s, uint32_t n, const Cliques &cl, const Instances &inst,
          const Tuning &t, uint32_t gl_buffer_size, PeelOut &out);

// Densest core, pruning and components; everything the flow stage needs.
struct CoreOut {
  std::vector<uint64_t> threshold;  // per instance k'
  std::vector<uint64_t> core_size;  // per instance
  std::vector<uint64_t> core_cliques;
  std::vector<uint64_t> pruned_edges;
  std::vector<uint32_t> n_components;
  // components with >= 1 clique, in (instance, smallest vertex) order
  uint32_t ncomp = 0;
  std::vector<uint32_t> comp_inst;    // instance of each component
  std::vector<uint32_t> comp_vbeg;    // [ncomp+1] local vertex ranges
  std::vector<uint64_t> comp_cbeg;    // [ncomp+1] clique ranges
  std::vector<uint32_t> comp_maxcore; // largest core number inside
  std::vector<uint32_t> comp_root;    // smallest vertex (problem id) of each component
  DBuf<uint32_t> vmap;      // [nv] original vertex of each local vertex
  DBuf<uint32_t> rec;       // [nc << rec_shift(k)] clique records: rec_slots(k)
                            // member slots (local vertex ids), then as many
                            // 32-bit flow words (written by the flow stage)
  DBuf<uint32_t> vcnet;     // [nv] component of each local vertex
  DBuf<uint64_t> vinc_off;  // [nv+1] incidence CSR: the cliques of each vertex
  DBuf<uint32_t> vinc;      // record indices as u32, or as u64 (pairs of words) when vinc_wide
  bool vinc_wide = false;
  mutable bool flows_zero = false;  // the records' flow words are still zero (the
                                    // first flow over them skips its reset pass)
  int mk_core = 0, mk_prune = 0;  // StageClock marks after the core and the pruning
};
struct StageClock;
void densest_core_and_components(cds_ctx *c, cudaStream_t s, const Dag &dag, const Cliques &cl,
                                 const PeelOut &pe, const Instances &inst, uint32_t k,
                                 CoreOut &out, bool need_networks, StageClock *clk = nullptr);

// Exact search over all component networks; per instance the answer set.
struct FlowAnswer {
  std::vector<uint64_t> num, den;          // per instance
  std::vector<std::vector<uint32_t>> set;  // per instance, original ids ascending
  std::vector<uint64_t> ub_num, ub_den;    // per instance: proven upper bound of the optimum
  // per component with cliques, in order: its instance, the starting lower
  // bound (the instance's densest whole component) and UB1
  std::vector<uint32_t> comp_inst;
  std::vector<double> comp_lb, comp_ub;
  uint32_t flows = 0;
  uint32_t early_stopped = 0;
};
void exact_search(cds_ctx *c, cudaStream_t s, const CoreOut &co, const Instances &inst,
                  uint32_t k, const cds_params &prm, const Tuning &t, FlowAnswer &ans);

}  // namespace cds
