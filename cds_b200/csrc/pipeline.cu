// pipeline.cu -- one solve over a problem (a graph, or a disjoint union of
// instance graphs sharing k), stage by stage, timed with device events.
//
// Replaces the stage sequence of the reference driver (cudaCode/main.cu:895-
// 1107) and CDS::DSD (cpuCode/c++/src/helpers.cpp:1422-1589).  Control stays
// on the device inside each stage; the host reads back only the scalars that
// size the next allocation.
#include "device_util.cuh"
#include "pipeline.h"

#include <algorithm>
#include <cstring>

namespace {

__global__ void k_union_adj(const uint32_t *__restrict__ src, uint64_t nnz, uint32_t shift,
                            uint32_t *__restrict__ dst) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i] + shift;
}

__global__ void k_union_off(const uint64_t *__restrict__ src, uint32_t n, uint64_t shift,
                            uint64_t *__restrict__ dst) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x)
    dst[v] = src[v] + shift;
}

__global__ void k_of_vertex(const uint32_t *__restrict__ vbeg, uint32_t ninst, uint32_t n,
                            uint32_t *__restrict__ of_vertex) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ninst;  // last i with vbeg[i] <= v
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (vbeg[mid] <= v) lo = mid;
      else hi = mid;
    }
    of_vertex[v] = lo;
  }
}

__global__ void k_inst_totals(const uint64_t *__restrict__ base, const uint32_t *__restrict__ vbeg,
                              uint32_t ninst, unsigned long long *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ninst; i += gridDim.x * blockDim.x)
    out[i] = base[vbeg[i + 1]] - base[vbeg[i]];
}

}  // namespace

namespace cds {

namespace {
struct PinnedArea {
  char *p = nullptr;
  size_t cap = 0, top = 0;
  bool tried = false;
  ~PinnedArea() {
    if (p) (void)cudaFreeHost(p);  // at thread exit; an error here has no one to report to
  }
};
thread_local PinnedArea t_pinned;  // one per host thread, freed when the thread ends
constexpr size_t PINNED_BYTES = 1 << 20;
}  // namespace

HostReads::HostReads(cudaStream_t s) : s_(s), base_(t_pinned.top) {}

HostReads::~HostReads() { t_pinned.top = base_; }

void HostReads::add_bytes(void *dst, const void *src, size_t bytes) {
  if (!t_pinned.tried) {
    t_pinned.tried = true;
    if (cudaHostAlloc(reinterpret_cast<void **>(&t_pinned.p), PINNED_BYTES, cudaHostAllocPortable) ==
        cudaSuccess)
      t_pinned.cap = PINNED_BYTES;
    else
      (void)cudaGetLastError();  // no pinned memory: every read goes direct
  }
  const size_t off = (t_pinned.top + 15) & ~size_t(15);
  if (bytes && off + bytes <= t_pinned.cap) {
    CDS_CUDA(cudaMemcpyAsync(t_pinned.p + off, src, bytes, cudaMemcpyDeviceToHost, s_));
    items_.push_back({dst, src, off, bytes});
    t_pinned.top = off + bytes;
  } else {
    items_.push_back({dst, src, SIZE_MAX, bytes});
  }
}

void HostReads::wait() {
  for (const Item &it : items_)
    if (it.off == SIZE_MAX && it.bytes)
      CDS_CUDA(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyDeviceToHost, s_));
  CDS_CUDA(cudaStreamSynchronize(s_));
  for (const Item &it : items_)
    if (it.off != SIZE_MAX) std::memcpy(it.dst, t_pinned.p + it.off, it.bytes);
  items_.clear();
  t_pinned.top = base_;
}

int StageClock::mark() {
  cudaEvent_t e;
  CDS_CUDA(cudaEventCreate(&e));
  ev.push_back(e);
  CDS_CUDA(cudaEventRecord(e, s));
  return (int)ev.size() - 1;
}
void StageClock::wait() {
  if (!ev.empty()) CDS_CUDA(cudaEventSynchronize(ev.back()));
}
double StageClock::ms(int a, int b) {
  float x = 0;
  CDS_CUDA(cudaEventElapsedTime(&x, ev[a], ev[b]));
  return x;
}
StageClock::~StageClock() {
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

void build_union(cds_ctx *c, cudaStream_t s, const std::vector<const cds_graph *> &gs,
                 UnionGraph &u) {
  uint32_t n = 0;
  uint64_t nnz = 0;
  u.inst.count = (uint32_t)gs.size();
  u.inst.h_vbeg.assign(gs.size() + 1, 0);
  for (size_t i = 0; i < gs.size(); i++) {
    if ((uint64_t)n + gs[i]->n >= 0xFFFFFFFFull) fail(CDS_ERR_OVERFLOW, "batch exceeds 2^32 vertices");
    n += gs[i]->n;
    nnz += gs[i]->nnz;
    u.inst.h_vbeg[i + 1] = n;
  }
  u.n = n;
  u.nnz = nnz;
  u.inst.vbeg = DBuf<uint32_t>(c, s, gs.size() + 1);
  CDS_CUDA(cudaMemcpyAsync(u.inst.vbeg.p, u.inst.h_vbeg.data(), (gs.size() + 1) * 4,
                           cudaMemcpyHostToDevice, s));
  // no wait: a copy from pageable memory has read its source when it returns
  if (gs.size() == 1) {
    u.off = gs[0]->d_off;
    u.adj = gs[0]->d_adj;
    return;
  }
  u.own_off = DBuf<uint64_t>(c, s, (size_t)n + 1);
  u.own_adj = DBuf<uint32_t>(c, s, nnz + 1);
  uint32_t vshift = 0;
  uint64_t eshift = 0;
  for (size_t i = 0; i < gs.size(); i++) {
    const cds_graph *g = gs[i];
    if (g->nnz)
      k_union_adj<<<c->sm_count * 2, 256, 0, s>>>(g->d_adj, g->nnz, vshift, u.own_adj.p + eshift);
    k_union_off<<<std::max(1u, (g->n + 256) / 256), 256, 0, s>>>(g->d_off, g->n, eshift,
                                                                  u.own_off.p + vshift);
    count_launch(2);
    vshift += g->n;
    eshift += g->nnz;
  }
  CDS_CUDA(cudaGetLastError());
  u.off = u.own_off.p;
  u.adj = u.own_adj.p;
  u.inst.of_vertex = DBuf<uint32_t>(c, s, (size_t)n + 1);
  if (n) {
    k_of_vertex<<<c->sm_count * 4, 256, 0, s>>>(u.inst.vbeg.p, u.inst.count, n, u.inst.of_vertex.p);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
}

// The densest core as the answer (no flow): per instance the level core
// {core >= L*} whose density |Psi_L*| / |V_L*| the peel found largest -- a
// real vertex set with that exact density -- and, as its proven upper bound
// of the optimum, the largest core number of the instance (every vertex of
// a densest set S lies in at least rho(S) of its cliques, so S sits inside
// the ceil(rho)-core).
void core_answer(cudaStream_t s, const PeelOut &pe, const UnionGraph &u, FlowAnswer &fa) {
  const uint32_t ninst = u.inst.count;
  fa.num = pe.best_num;
  fa.den = pe.best_den;
  fa.set.assign(ninst, {});
  fa.ub_num.assign(ninst, 0);
  fa.ub_den.assign(ninst, 1);
  for (uint32_t i = 0; i < ninst; i++) fa.ub_num[i] = pe.inst_max_core[i];
  if (u.n == 0) return;
  std::vector<uint32_t> core(u.n);
  {
    HostReads r(s);
    r.add(core.data(), pe.core.p, u.n);
    r.wait();
  }
  for (uint32_t i = 0; i < ninst; i++) {
    if (!pe.best_num[i]) {  // no cliques: the empty answer, as the exact search gives
      fa.num[i] = fa.den[i] = 0;
      continue;
    }
    const uint32_t b = u.inst.h_vbeg[i], e = u.inst.h_vbeg[i + 1];
    for (uint32_t v = b; v < e; v++)
      if (core[v] >= pe.best_level[i]) fa.set[i].push_back(v - b);
    if (fa.set[i].size() != pe.best_den[i]) fail(CDS_ERR_CUDA, "densest core size does not match its level");
  }
}

void run_problem(cds_ctx *c, cudaStream_t s, UnionGraph &u, const cds_params &prm,
                 std::vector<ProblemResult> &res, const CountHook *on_count) {
  const uint32_t k = prm.k;
  if (k < 2 || k > CDS_MAX_K) fail(CDS_ERR_INPUT, "k must be in [2, 16]");
  if (prm.search > CDS_SEARCH_CORE) fail(CDS_ERR_INPUT, "search must be 0, 1 or 2");
  const bool core_only = prm.search == CDS_SEARCH_CORE;
  const Tuning &t = c->tune[k];
  const uint32_t ninst = u.inst.count;
  res.assign(ninst, ProblemResult{});
  StageClock clk(s);
  double tms[CDS_T_COUNT] = {0};
  const int m0 = clk.mark();

  Dag dag;
  dag.deg = DBuf<uint32_t>(c, s, 0);
  dag.outdeg = DBuf<uint32_t>(c, s, 0);
  dag.off = DBuf<uint64_t>(c, s, 0);
  dag.adj = DBuf<uint32_t>(c, s, 0);
  build_dag(c, s, u.off, u.adj, u.n, dag);
  const int m1 = clk.mark();

  Cliques cl;
  list_cliques(c, s, dag, k, true, t, cl, on_count);
  const int m2 = clk.mark();

  PeelOut pe;
  peel(c, s, u.n, cl, u.inst, t, prm.gl_buffer_size, pe);
  const int m3 = clk.mark();

  CoreOut co;
  densest_core_and_components(c, s, dag, cl, pe, u.inst, k, co, !core_only, &clk);
  const int m4 = clk.mark();

  // per-instance clique totals
  std::vector<unsigned long long> tot(ninst);
  {
    DBuf<unsigned long long> d(c, s, ninst);
    k_inst_totals<<<std::max(1u, (ninst + 255) / 256), 256, 0, s>>>(cl.base.p, u.inst.vbeg.p, ninst, d.p);
    count_launch();
    CDS_CUDA(cudaGetLastError());
    HostReads r(s);
    r.add(tot.data(), d.p, ninst);
    r.wait();
  }
  // the clique store and incidence lists are no longer needed
  cl.members.release();

  FlowAnswer fa;
  if (core_only) core_answer(s, pe, u, fa);
  else exact_search(c, s, co, u.inst, k, prm, t, fa);
  const int m5 = clk.mark();
  clk.wait();
  tms[CDS_T_DAG] = clk.ms(m0, m1);
  tms[CDS_T_LIST] = clk.ms(m1, m2);
  tms[CDS_T_PEEL] = clk.ms(m2, m3);
  tms[CDS_T_CORE] = clk.ms(m3, co.mk_core);
  tms[CDS_T_PRUNE] = clk.ms(co.mk_core, co.mk_prune);
  tms[CDS_T_COMPONENTS] = clk.ms(co.mk_prune, m4);
  tms[CDS_T_EXACT] = clk.ms(m4, m5);
  double total = 0;
  for (int i = 0; i < CDS_T_TOTAL; i++) total += tms[i];
  tms[CDS_T_TOTAL] = total;

  for (uint32_t i = 0; i < ninst; i++) {
    ProblemResult &r = res[i];
    r.total_cliques = tot[i];
    r.max_core = pe.inst_max_core[i];
    r.core_threshold = co.threshold[i];
    r.core_num = pe.best_num[i];
    r.core_den = pe.best_den[i];
    r.core_size = co.core_size[i];
    r.core_cliques = co.core_cliques[i];
    r.pruned_edges = co.pruned_edges[i];
    r.n_components = co.n_components[i];
    r.flows = fa.flows;
    r.early_stopped = fa.early_stopped;
    r.num = fa.num[i];
    r.den = fa.den[i];
    r.vertices = std::move(fa.set[i]);
    r.ub_num = fa.ub_num[i];
    r.ub_den = fa.ub_den[i];
    for (size_t j = 0; j < fa.comp_inst.size(); j++)
      if (fa.comp_inst[j] == i) {
        r.bound_lb.push_back(fa.comp_lb[j]);
        r.bound_ub.push_back(fa.comp_ub[j]);
      }
    std::memcpy(r.t_ms, tms, sizeof(tms));
    r.levels = pe.inst_levels[i];
  }
}

}  // namespace cds
