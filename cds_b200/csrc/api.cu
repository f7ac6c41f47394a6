// api.cu -- the C ABI (include/cds.h): contexts, device memory pool, graphs,
// stage entry points, single and batched solves.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>

#include "cds_gen.h"
#include "device_util.cuh"
#include "pipeline.h"

namespace cds {

std::atomic<uint64_t> g_launches{0};

void fail(cds_status s, const std::string &msg) { throw Error{s, msg}; }

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  const cds_status s = (e == cudaErrorMemoryAllocation) ? CDS_ERR_OOM : CDS_ERR_CUDA;
  fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

void *dalloc_bytes(cds_ctx *c, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return nullptr;
  bytes = (bytes + 255) & ~size_t(255);
  const uint64_t now = c->in_use.fetch_add(bytes) + bytes;
  if (now > c->budget) {
    c->in_use.fetch_sub(bytes);
    fail(CDS_ERR_OOM, "device memory budget exceeded (" + std::to_string(now) + " > " +
                          std::to_string(c->budget) + " bytes)");
  }
  void *p = nullptr;
  const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, c->pool, s);
  if (e != cudaSuccess) {
    c->in_use.fetch_sub(bytes);
    cudaGetLastError();
    fail(CDS_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  uint64_t pk = c->peak.load();
  while (now > pk && !c->peak.compare_exchange_weak(pk, now)) {
  }
  std::lock_guard<std::mutex> g(c->mu);
  c->sizes[p] = bytes;
  return p;
}

void dfree(cds_ctx *c, void *p, cudaStream_t s) {
  size_t bytes = 0;
  {
    std::lock_guard<std::mutex> g(c->mu);
    auto it = c->sizes.find(p);
    if (it != c->sizes.end()) {
      bytes = it->second;
      c->sizes.erase(it);
    }
  }
  cudaFreeAsync(p, s);
  c->in_use.fetch_sub(bytes);
}

namespace {

// rows strictly ascending, no self-loops, ids < n, every arc has its reverse
__global__ void k_check_csr(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                            uint32_t n, uint32_t *__restrict__ bad) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = off[v], e = off[v + 1];
    uint32_t flag = 0;
    for (uint64_t i = b + lane_id(); i < e; i += 32) {
      const uint32_t w = adj[i];
      if (w >= n || w == v || (i > b && adj[i - 1] >= w)) {
        flag = 1;
        continue;
      }
      uint64_t lo = off[w], hi = off[w + 1];
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (adj[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      if (lo >= off[w + 1] || adj[lo] != v) flag = 1;
    }
    if (__any_sync(CDS_FULL, flag) && lane_id() == 0) atomicOr(bad, 1u);
  }
}

}  // namespace

PinnedHost::PinnedHost(size_t bytes) {
  if (cudaHostAlloc(reinterpret_cast<void **>(&p), bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
    (void)cudaGetLastError();
    p = nullptr;
    fail(CDS_ERR_OOM, "pinned host allocation failed");
  }
}
PinnedHost::~PinnedHost() {
  if (p) (void)cudaFreeHost(p);
}

cds_status graph_upload(cds_ctx *c, cudaStream_t s, const uint64_t *off, const uint32_t *adj,
                        uint32_t n, cds_graph **out) {
  if (off[0] != 0) fail(CDS_ERR_INPUT, "off[0] must be 0");
  for (uint32_t v = 0; v < n; v++)
    if (off[v + 1] < off[v]) fail(CDS_ERR_INPUT, "offsets must not decrease");
  cds_graph *g = new cds_graph();
  g->ctx = c;
  g->n = n;
  g->nnz = off[n];
  try {
    g->d_off = (uint64_t *)dalloc_bytes(c, ((size_t)n + 1) * 8, s);
    g->d_adj = (uint32_t *)dalloc_bytes(c, (size_t)g->nnz * 4 + 16, s);
    CDS_CUDA(cudaMemcpyAsync(g->d_off, off, ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, s));
    if (g->nnz) CDS_CUDA(cudaMemcpyAsync(g->d_adj, adj, (size_t)g->nnz * 4, cudaMemcpyHostToDevice, s));
    DBuf<uint32_t> bad(c, s, 1);
    bad.zero();
    if (n) {
      k_check_csr<<<c->sm_count * 8, 256, 0, s>>>(g->d_off, g->d_adj, n, bad.p);
      count_launch();
      CDS_CUDA(cudaGetLastError());
    }
    if (d2h(bad.p, s))
      fail(CDS_ERR_INPUT, "CSR must be symmetric with ascending rows, ids < n and no self-loops");
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; v++) maxd = std::max<uint32_t>(maxd, (uint32_t)(off[v + 1] - off[v]));
    g->max_degree = maxd;
  } catch (...) {
    if (g->d_off) dfree(c, g->d_off, s);
    if (g->d_adj) dfree(c, g->d_adj, s);
    delete g;
    throw;
  }
  *out = g;
  return CDS_OK;
}

void fill_result(const ProblemResult &r, cds_result *out) {
  std::memset(out, 0, sizeof(*out));
  out->num = r.num;
  out->den = r.den;
  out->total_cliques = r.total_cliques;
  out->max_core = r.max_core;
  out->core_threshold = r.core_threshold;
  out->core_num = r.core_num;
  out->core_den = r.core_den;
  out->core_size = r.core_size;
  out->core_cliques = r.core_cliques;
  out->pruned_edges = r.pruned_edges;
  out->n_components = r.n_components;
  out->flows = r.flows;
  out->early_stopped = r.early_stopped;
  out->peel_levels = r.levels;
  std::memcpy(out->t_ms, r.t_ms, sizeof(out->t_ms));
  out->size = r.vertices.size();
  out->ub_num = r.ub_num;
  out->ub_den = r.ub_den;
  if (out->size) {
    out->vertices = (uint32_t *)std::malloc(out->size * sizeof(uint32_t));
    if (!out->vertices) fail(CDS_ERR_OOM, "host allocation failed");
    std::memcpy(out->vertices, r.vertices.data(), out->size * sizeof(uint32_t));
  }
  const size_t nb = r.bound_lb.size();
  if (nb) {
    out->bound_lb = (double *)std::malloc(nb * sizeof(double));
    out->bound_ub = (double *)std::malloc(nb * sizeof(double));
    if (!out->bound_lb || !out->bound_ub) {
      std::free(out->vertices);
      std::free(out->bound_lb);
      std::free(out->bound_ub);
      out->vertices = nullptr;
      out->bound_lb = out->bound_ub = nullptr;
      fail(CDS_ERR_OOM, "host allocation failed");
    }
    std::memcpy(out->bound_lb, r.bound_lb.data(), nb * sizeof(double));
    std::memcpy(out->bound_ub, r.bound_ub.data(), nb * sizeof(double));
    out->n_bounds = (uint32_t)nb;
  }
}

}  // namespace cds

using namespace cds;

namespace {

template <class F>
cds_status guarded(cds_ctx *c, F &&f) {
  try {
    f();
    return CDS_OK;
  } catch (const Error &e) {
    if (c) {
      std::lock_guard<std::mutex> g(c->mu);
      c->err = e.msg;
    }
    return e.status;
  } catch (const std::bad_alloc &) {
    if (c) {
      std::lock_guard<std::mutex> g(c->mu);
      c->err = "host allocation failed";
    }
    return CDS_ERR_OOM;
  } catch (const std::exception &e) {
    if (c) {
      std::lock_guard<std::mutex> g(c->mu);
      c->err = e.what();
    }
    return CDS_ERR_STATE;
  }
}

void check_graph(cds_ctx *c, const cds_graph *g) {
  if (!g) fail(CDS_ERR_INPUT, "graph is NULL");
  if (g->ctx != c) fail(CDS_ERR_INPUT, "graph belongs to another context");
}

}  // namespace

extern "C" {

uint64_t cds_kernel_launches(void) { return g_launches.load(); }

cds_status cds_profile(cds_ctx *c, int on) {
  if (!c) return CDS_ERR_INPUT;
  c->prof = on != 0;
  return CDS_OK;
}

cds_status cds_profile_read(cds_ctx *c, char *buf, size_t len) {
  if (!c || !buf) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    std::vector<ProfEvent> ev;
    {
      std::lock_guard<std::mutex> g(c->mu);
      ev.swap(c->prof_pending);
    }
    for (auto &e : ev) {
      CDS_CUDA(cudaEventSynchronize(e.b));
      float ms = 0;
      CDS_CUDA(cudaEventElapsedTime(&ms, e.a, e.b));
      auto &slot = c->prof_done[e.name];
      slot.first += 1;
      slot.second += ms;
      cudaEventDestroy(e.a);
      cudaEventDestroy(e.b);
    }
    std::string out = "{";
    bool first = true;
    for (auto &kv : c->prof_done) {
      char tmp[256];
      std::snprintf(tmp, sizeof(tmp), "%s\"%s\": [%llu, %.6f]", first ? "" : ", ", kv.first.c_str(),
                    (unsigned long long)kv.second.first, kv.second.second);
      out += tmp;
      first = false;
    }
    out += "}";
    if (out.size() + 1 > len) fail(CDS_ERR_INPUT, "profile buffer too small");
    std::memcpy(buf, out.c_str(), out.size() + 1);
    c->prof_done.clear();
  });
}

const char *cds_version(void) { return "cds-b200 1.0 (sm_100a)"; }

const char *cds_status_string(cds_status s) {
  switch (s) {
    case CDS_OK: return "ok";
    case CDS_ERR_OOM: return "out of device memory";
    case CDS_ERR_OVERFLOW: return "count overflow";
    case CDS_ERR_TIMEOUT: return "device iteration budget exhausted";
    case CDS_ERR_INPUT: return "invalid input";
    case CDS_ERR_CUDA: return "CUDA error";
    case CDS_ERR_STATE: return "invalid state";
    case CDS_ERR_NOT_READY: return "not ready";
  }
  return "unknown status";
}

cds_status cds_create(const cds_config *cfg, cds_ctx **out) {
  if (!out) return CDS_ERR_INPUT;
  *out = nullptr;
  if (cfg && cfg->streams > CDS_MAX_INFLIGHT) return CDS_ERR_INPUT;
  cds_ctx *c = new (std::nothrow) cds_ctx();
  if (!c) return CDS_ERR_OOM;
  const cds_status st = guarded(c, [&] {
    const int dev = cfg ? cfg->device : 0;
    int ndev = 0;
    CDS_CUDA(cudaGetDeviceCount(&ndev));
    if (dev < 0 || dev >= ndev) fail(CDS_ERR_INPUT, "no such CUDA device");
    CDS_CUDA(cudaSetDevice(dev));
    cudaDeviceProp prop;
    CDS_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) fail(CDS_ERR_CUDA, "libcds is built for sm_100a (B200)");
    int coop = 0;
    CDS_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) fail(CDS_ERR_CUDA, "device lacks cooperative launch");
    c->device = dev;
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    CDS_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->flags = cfg ? cfg->flags : 0u;
    const uint32_t nw = (cfg && cfg->streams) ? cfg->streams : 4;
    for (uint32_t i = 0; i < nw; i++) {
      cudaStream_t w;
      CDS_CUDA(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
      c->workers.push_back(w);
    }
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = dev;
    CDS_CUDA(cudaMemPoolCreate(&c->pool, &pp));
    // per-k launch shapes measured on R-MAT graphs (cds_autotune refines
    // them): for k >= 3 roots of out-degree above 32 go to block teams, whose
    // 512 threads share a dense neighbourhood's pairs, more push/relabel
    // rounds pass between global relabels, and peel items hold up to 1,024
    // incidences (fewer hub flushes; k = 2 keeps 512); for k <= 3 peel items
    // go in ascending clique-degree order (for k >= 4 that costs sweeps)
    for (uint32_t k = 0; k <= CDS_MAX_K; k++) {
      if (k >= 3) c->tune[k].list_warp_dmax = 32;
      if (k >= 3) c->tune[k].flow_rounds = 32;
      if (k >= 3) c->tune[k].peel_chunk = 1024;
      if (k <= 3) c->tune[k].peel_order = 1;  // fewer, cheaper sweeps for k = 2, 3
      // k >= 4: half the peel items dealt round-robin, the rest by a counter
      // (R-MAT-18 k = 4: 736 -> 640 ms; R-MAT-14 k = 4: 2.25 -> 1.82 ms; at
      // k = 2, 3 the counter costs more than the balance gains)
      if (k >= 4) c->tune[k].peel_static = 50;
    }
    uint64_t keep = ~0ull;  // keep freed blocks cached in the pool
    CDS_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    size_t fr = 0, tot = 0;
    CDS_CUDA(cudaMemGetInfo(&fr, &tot));
    c->budget = (cfg && cfg->mem_budget) ? cfg->mem_budget : (uint64_t)(0.9 * (double)fr);
  });
  if (st != CDS_OK) {
    cds_destroy(c);
    return st;
  }
  *out = c;
  return CDS_OK;
}

void cds_destroy(cds_ctx *c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (cudaStream_t w : c->workers) {
    cudaStreamSynchronize(w);
    cudaStreamDestroy(w);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->pool) cudaMemPoolDestroy(c->pool);
  delete c;
}

const char *cds_last_error(const cds_ctx *c) { return c ? c->err.c_str() : "no context"; }

cds_status cds_mem_usage(const cds_ctx *c, uint64_t *in_use, uint64_t *peak) {
  if (!c) return CDS_ERR_INPUT;
  if (in_use) *in_use = c->in_use.load();
  if (peak) *peak = c->peak.load();
  return CDS_OK;
}

cds_status cds_graph_from_csr(cds_ctx *c, const uint64_t *off, const uint32_t *adj, uint32_t n,
                              cds_graph **out) {
  if (!c || !off || !out || (n && off[n] && !adj)) return CDS_ERR_INPUT;
  return guarded(c, [&] { graph_upload(c, c->stream, off, adj, n, out); });
}

cds_status cds_graph_load_file(cds_ctx *c, const char *path, cds_graph **out) {
  if (!c || !path || !out) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    cudaStream_t s = c->stream;
    FILE *f = std::fopen(path, "rb");
    if (!f) fail(CDS_ERR_INPUT, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) {
      std::fclose(f);
      fail(CDS_ERR_INPUT, std::string("cannot read ") + path);
    }
    // the bytes go through pinned host memory (one read, one copy)
    PinnedHost buf((size_t)sz + 1);
    const size_t got = sz ? std::fread(buf.p, 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if (got != (size_t)sz) fail(CDS_ERR_INPUT, std::string("cannot read ") + path);
    if ((size_t)sz >= sizeof(cds_csr_header) && std::memcmp(buf.p, CDS_CSR_MAGIC, 8) == 0) {
      // binary CSR cache: the arrays as they are (the upload checks them)
      cds_csr_header h;
      std::memcpy(&h, buf.p, sizeof(h));
      if (h.version != 1 || h.n >= 0xFFFFFFFFull ||
          (uint64_t)sz != sizeof(h) + 8 * (h.n + 1) + 4 * h.nnz)
        fail(CDS_ERR_INPUT, std::string("malformed binary CSR file ") + path);
      const uint64_t *off = reinterpret_cast<const uint64_t *>(buf.p + sizeof(h));
      if (off[h.n] != h.nnz) fail(CDS_ERR_INPUT, std::string("malformed binary CSR file ") + path);
      const uint32_t *adj = reinterpret_cast<const uint32_t *>(buf.p + sizeof(h) + 8 * (h.n + 1));
      graph_upload(c, s, off, adj, (uint32_t)h.n, out);
      return;
    }
    // adjacency-list text, parsed on the device
    DBuf<uint8_t> txt(c, s, (size_t)sz + 1);
    if (sz) CDS_CUDA(cudaMemcpyAsync(txt.p, buf.p, (size_t)sz, cudaMemcpyHostToDevice, s));
    parse_adjlist_device(c, s, txt.p, (uint64_t)sz, out);
  });
}

cds_status cds_graph_info(const cds_graph *g, uint32_t *n, uint64_t *m, uint32_t *max_degree) {
  if (!g) return CDS_ERR_INPUT;
  if (n) *n = g->n;
  if (m) *m = g->nnz / 2;
  if (max_degree) *max_degree = g->max_degree;
  return CDS_OK;
}

cds_status cds_graph_download(const cds_graph *g, uint64_t *off, uint32_t *adj) {
  if (!g || !off || (g->nnz && !adj)) return CDS_ERR_INPUT;
  cds_ctx *c = g->ctx;
  return guarded(c, [&] {
    CDS_CUDA(cudaMemcpyAsync(off, g->d_off, ((size_t)g->n + 1) * 8, cudaMemcpyDeviceToHost, c->stream));
    if (g->nnz) CDS_CUDA(cudaMemcpyAsync(adj, g->d_adj, (size_t)g->nnz * 4, cudaMemcpyDeviceToHost, c->stream));
    CDS_CUDA(cudaStreamSynchronize(c->stream));
  });
}

void cds_graph_free(cds_graph *g) {
  if (!g) return;
  cds_ctx *c = g->ctx;
  if (g->d_off) dfree(c, g->d_off, c->stream);
  if (g->d_adj) dfree(c, g->d_adj, c->stream);
  cudaStreamSynchronize(c->stream);
  delete g;
}

cds_status cds_list_cliques(cds_ctx *c, cds_graph *g, uint32_t k, uint32_t p_size,
                            uint32_t cp_size, uint64_t *count, uint64_t *clique_degree) {
  (void)p_size;
  (void)cp_size;
  if (!c) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    check_graph(c, g);
    cudaStream_t s = c->stream;
    Dag dag;
    dag.deg = DBuf<uint32_t>(c, s, 0);
    dag.outdeg = DBuf<uint32_t>(c, s, 0);
    dag.off = DBuf<uint64_t>(c, s, 0);
    dag.adj = DBuf<uint32_t>(c, s, 0);
    build_dag(c, s, g->d_off, g->d_adj, g->n, dag);
    Cliques cl;
    list_cliques(c, s, dag, k, false, c->tune[k < 2 ? 2 : (k > CDS_MAX_K ? CDS_MAX_K : k)], cl);
    if (count) *count = cl.count;
    if (clique_degree && g->n)
      CDS_CUDA(cudaMemcpyAsync(clique_degree, cl.cdeg64.p, (size_t)g->n * 8, cudaMemcpyDeviceToHost, s));
    CDS_CUDA(cudaStreamSynchronize(s));
  });
}

cds_status cds_clique_core(cds_ctx *c, cds_graph *g, uint32_t k, uint32_t gl_buffer_size,
                           uint64_t *core, uint64_t *max_core, uint64_t *count) {
  if (!c) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    check_graph(c, g);
    if (k < 2 || k > CDS_MAX_K) fail(CDS_ERR_INPUT, "k must be in [2, 16]");
    cudaStream_t s = c->stream;
    UnionGraph u;
    build_union(c, s, {g}, u);
    Dag dag;
    dag.deg = DBuf<uint32_t>(c, s, 0);
    dag.outdeg = DBuf<uint32_t>(c, s, 0);
    dag.off = DBuf<uint64_t>(c, s, 0);
    dag.adj = DBuf<uint32_t>(c, s, 0);
    build_dag(c, s, u.off, u.adj, u.n, dag);
    Cliques cl;
    list_cliques(c, s, dag, k, true, c->tune[k], cl);
    PeelOut pe;
    peel(c, s, u.n, cl, u.inst, c->tune[k], gl_buffer_size, pe);
    if (count) *count = cl.count;
    if (max_core) *max_core = pe.max_core;
    if (core && g->n) {
      std::vector<uint32_t> h(g->n);
      CDS_CUDA(cudaMemcpyAsync(h.data(), pe.core.p, (size_t)g->n * 4, cudaMemcpyDeviceToHost, s));
      CDS_CUDA(cudaStreamSynchronize(s));
      for (uint32_t v = 0; v < g->n; v++) core[v] = h[v];
    }
    CDS_CUDA(cudaStreamSynchronize(s));
  });
}

cds_status cds_densest_core(cds_ctx *c, cds_graph *g, uint32_t k, uint64_t *threshold,
                            uint64_t *num, uint64_t *den, uint8_t *in_core) {
  if (!c) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    check_graph(c, g);
    if (k < 2 || k > CDS_MAX_K) fail(CDS_ERR_INPUT, "k must be in [2, 16]");
    cudaStream_t s = c->stream;
    UnionGraph u;
    build_union(c, s, {g}, u);
    Dag dag;
    dag.deg = DBuf<uint32_t>(c, s, 0);
    dag.outdeg = DBuf<uint32_t>(c, s, 0);
    dag.off = DBuf<uint64_t>(c, s, 0);
    dag.adj = DBuf<uint32_t>(c, s, 0);
    build_dag(c, s, u.off, u.adj, u.n, dag);
    Cliques cl;
    list_cliques(c, s, dag, k, true, c->tune[k], cl);
    PeelOut pe;
    peel(c, s, u.n, cl, u.inst, c->tune[k], 0, pe);
    const uint64_t bn = pe.best_num[0], bd = pe.best_den[0];
    const uint64_t t = (bd && bn) ? (bn + bd - 1) / bd : 0;
    if (threshold) *threshold = t;
    if (num) *num = bn;
    if (den) *den = bd;
    if (in_core && g->n) {
      std::vector<uint32_t> h(g->n);
      CDS_CUDA(cudaMemcpyAsync(h.data(), pe.core.p, (size_t)g->n * 4, cudaMemcpyDeviceToHost, s));
      CDS_CUDA(cudaStreamSynchronize(s));
      for (uint32_t v = 0; v < g->n; v++) in_core[v] = t > 0 && (uint64_t)h[v] >= t;
    }
  });
}

cds_status cds_components(cds_ctx *c, cds_graph *g, uint32_t k, uint64_t *core_cliques,
                          uint64_t *pruned_edges, uint32_t *count, uint32_t *first, uint64_t *size,
                          uint64_t *cliques, size_t cap) {
  if (!c) return CDS_ERR_INPUT;
  return guarded(c, [&] {
    check_graph(c, g);
    if (k < 2 || k > CDS_MAX_K) fail(CDS_ERR_INPUT, "k must be in [2, 16]");
    cudaStream_t s = c->stream;
    UnionGraph u;
    build_union(c, s, {g}, u);
    Dag dag;
    dag.deg = DBuf<uint32_t>(c, s, 0);
    dag.outdeg = DBuf<uint32_t>(c, s, 0);
    dag.off = DBuf<uint64_t>(c, s, 0);
    dag.adj = DBuf<uint32_t>(c, s, 0);
    build_dag(c, s, u.off, u.adj, u.n, dag);
    Cliques cl;
    list_cliques(c, s, dag, k, true, c->tune[k], cl);
    PeelOut pe;
    peel(c, s, u.n, cl, u.inst, c->tune[k], 0, pe);
    CoreOut co;
    densest_core_and_components(c, s, dag, cl, pe, u.inst, k, co, true, nullptr);
    CDS_CUDA(cudaStreamSynchronize(s));
    if (core_cliques) *core_cliques = co.core_cliques[0];
    if (pruned_edges) *pruned_edges = co.pruned_edges[0];
    if (count) *count = co.ncomp;
    const size_t m = std::min<size_t>(cap, co.ncomp);
    for (size_t i = 0; i < m; i++) {
      if (first) first[i] = co.comp_root[i];
      if (size) size[i] = co.comp_vbeg[i + 1] - co.comp_vbeg[i];
      if (cliques) cliques[i] = co.comp_cbeg[i + 1] - co.comp_cbeg[i];
    }
  });
}

cds_status cds_solve(cds_ctx *c, cds_graph *g, const cds_params *params, cds_result *result) {
  if (!c || !params || !result) return CDS_ERR_INPUT;
  std::memset(result, 0, sizeof(*result));
  return guarded(c, [&] {
    check_graph(c, g);
    UnionGraph u;
    build_union(c, c->stream, {g}, u);
    std::vector<ProblemResult> res;
    run_problem(c, c->stream, u, *params, res);
    fill_result(res[0], result);
  });
}

void cds_result_free(cds_result *r) {
  if (!r) return;
  std::free(r->vertices);
  std::free(r->bound_lb);
  std::free(r->bound_ub);
  r->vertices = nullptr;
  r->bound_lb = r->bound_ub = nullptr;
  r->size = 0;
  r->n_bounds = 0;
}

cds_status cds_solve_batch(cds_ctx *c, const cds_job *jobs, size_t n, cds_result *results) {
  if (!c || (n && (!jobs || !results))) return CDS_ERR_INPUT;
  for (size_t i = 0; i < n; i++) std::memset(&results[i], 0, sizeof(cds_result));
  return guarded(c, [&] {
    // one problem per (k, search, early_stop) group; groups run on worker streams
    std::vector<std::vector<size_t>> groups;
    std::vector<cds_params> gp;
    for (size_t i = 0; i < n; i++) {
      check_graph(c, jobs[i].graph);
      const cds_params &p = jobs[i].params;
      size_t gi = 0;
      for (; gi < gp.size(); gi++)
        if (gp[gi].k == p.k && gp[gi].search == p.search && gp[gi].early_stop == p.early_stop) break;
      if (gi == gp.size()) {
        gp.push_back(p);
        groups.emplace_back();
      }
      groups[gi].push_back(i);
    }
    for (size_t gi = 0; gi < groups.size(); gi++) {
      cudaStream_t s = c->workers.empty() ? c->stream : c->workers[gi % c->workers.size()];
      std::vector<const cds_graph *> gs;
      for (size_t i : groups[gi]) gs.push_back(jobs[i].graph);
      UnionGraph u;
      build_union(c, s, gs, u);
      std::vector<ProblemResult> res;
      run_problem(c, s, u, gp[gi], res);
      for (size_t j = 0; j < groups[gi].size(); j++) fill_result(res[j], &results[groups[gi][j]]);
    }
  });
}

}  // extern "C"
