// server.cpp -- request loop with continuous batching (cds_server_* in cds.h).
//
// The reference has no serving mode; this is new.  Requests are queued by
// cds_submit (a resident graph) or cds_submit_csr (a host CSR the worker
// uploads).  Up to max_inflight worker threads, one per context stream,
// each take the oldest pending request and, with it, later pending requests
// of the same k and size class (up to max_batch), run them as one batched
// problem, and publish every result as soon as that problem is solved.  A
// request that arrives while batches run is taken by the next worker that
// frees up, so work from different arrivals overlaps on the device.
//
// Size classes keep small requests from waiting on large ones: a request
// whose graph has at least LARGE_ARCS arcs runs alone, and while there are
// two or more workers at least one of them never takes a large request.
//
// Admission by memory, in two steps.  Before a batch starts it reserves a
// bound on what its graphs, DAGs and listing work arrays take.  After the
// listing's count pass, when |Psi| is known and before anything sized by it
// is allocated, the worker reserves what the clique store, the peel's
// incidence streams and the flow networks can take, waiting while that does
// not fit what the budget has left and another batch is running.  A batch
// that still runs out of device memory is split: each of its requests is
// queued again to run alone, and only a request that fails alone reports
// its error (CDS_ERR_OOM or another).  A request whose host CSR is malformed
// is answered with CDS_ERR_INPUT before its batch runs.  Results are kept
// until polled.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>

#include "pipeline.h"

namespace {

using Clock = std::chrono::steady_clock;

// Graphs with at least this many directed arcs are solved one per batch.
constexpr uint64_t LARGE_ARCS = 1ull << 20;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct cds_server {
  cds_ctx *ctx = nullptr;
  cds_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_mem;
  struct Req {
    uint64_t ticket;
    cds_graph *g;              // resident graph, or null for a host CSR
    const uint64_t *off;       // host CSR (cds_submit_csr)
    const uint32_t *adj;
    uint32_t n;
    uint64_t nnz;
    cds_params p;
    uint64_t est;              // reservation before the count
    bool alone;                // run as a batch of one (after a failed batch)
    Clock::time_point submitted;
  };
  std::deque<Req> pending;
  struct Done {
    cds_status st;
    cds::ProblemResult r;
    double queue_ms, service_ms;
  };
  std::map<uint64_t, Done> done;
  std::map<uint64_t, bool> inflight;  // tickets a worker is solving
  uint64_t next_ticket = 1;
  uint64_t mem_reserved = 0;
  uint64_t budget = 0;
  uint32_t running = 0;       // workers inside a batch
  uint32_t waiting_mem = 0;   // of those, waiting for a memory reservation
  uint32_t large_running = 0;
  uint32_t nworkers = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
};

namespace {

bool is_large(const cds_server::Req &r) { return r.nnz >= LARGE_ARCS; }

// Device bytes a request takes before its clique count is known: its graph
// (when uploaded), DAG, listing work arrays and per-vertex state.
uint64_t pre_count_bytes(uint64_t n, uint64_t nnz, bool upload) {
  uint64_t b = 96 * (n + 1) + 8 * nnz;
  if (upload) b += 8 * (n + 1) + 4 * nnz;
  return b + (1u << 20);
}

// Device bytes sized by |Psi|: the clique store (4k per clique), and the
// larger of the peel's incidence streams (the layout peel.cu picks) and the
// flow networks' members, incidences and flow state (at most 12k + 4 per
// clique); the estimate used for admission once the count is known.
uint64_t post_count_bytes(uint64_t cliques, uint32_t k, uint64_t n) {
  uint64_t peel;
  if (k <= 4 && n <= 65536) peel = 2ull * k * (k - 1);
  else if ((k == 3 || k == 4) && n <= (1u << 21)) peel = 8ull * k;
  else if (k <= 4) peel = 4ull * k * (k - 1);
  else peel = 4ull * k;
  const uint64_t flow = 12ull * k + 4;
  return cliques * (4ull * k + (peel > flow ? peel : flow)) + (16u << 20);
}

void publish(cds_server *s, const std::vector<cds_server::Req> &batch, cds_status st,
             std::vector<cds::ProblemResult> &res, Clock::time_point started) {
  const Clock::time_point now = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  for (size_t i = 0; i < batch.size(); i++) {
    cds_server::Done d;
    d.st = st;
    if (st == CDS_OK) d.r = std::move(res[i]);
    d.queue_ms = ms_between(batch[i].submitted, started);
    d.service_ms = ms_between(started, now);
    s->done[batch[i].ticket] = std::move(d);
    s->inflight.erase(batch[i].ticket);
  }
}

void worker_main(cds_server *s, size_t wi) {
  cds_ctx *c = s->ctx;
  cudaStream_t stream = c->workers.empty() ? c->stream : c->workers[wi % c->workers.size()];
  cudaSetDevice(c->device);
  for (;;) {
    std::vector<cds_server::Req> batch;
    uint64_t est = 0;
    bool large = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // the first pending request this worker may take: a large one only
      // while another worker stays free for small ones
      // index of the first pending request this worker may take: a large
      // one only while another worker stays free for small ones
      auto pick = [&]() -> size_t {
        for (size_t i = 0; i < s->pending.size(); i++) {
          const cds_server::Req &r = s->pending[i];
          if (!is_large(r) || s->nworkers < 2 || s->large_running + 1 < s->nworkers) return i;
        }
        return s->pending.size();
      };
      s->cv_work.wait(lk, [&] { return pick() < s->pending.size() || (s->stopping && s->pending.empty()); });
      const size_t first = pick();
      if (first >= s->pending.size()) return;  // stopping, and nothing is left
      // the head request, then later ones of its k, search mode, early stop
      // and size class while they fit (positions, not iterators: erasing
      // inside a deque moves its elements)
      const cds_server::Req head = s->pending[first];
      s->pending.erase(s->pending.begin() + (ptrdiff_t)first);
      batch.push_back(head);
      est = head.est;
      large = is_large(head);
      const uint32_t cap = (large || head.alone) ? 1u : (s->cfg.max_batch ? s->cfg.max_batch : 64u);
      for (size_t i = first; i < s->pending.size() && batch.size() < cap;) {
        const cds_server::Req &r = s->pending[i];
        if (r.p.k == head.p.k && r.p.search == head.p.search && r.p.early_stop == head.p.early_stop &&
            !r.alone && is_large(r) == large && s->mem_reserved + est + r.est <= s->budget) {
          est += r.est;
          batch.push_back(r);
          s->pending.erase(s->pending.begin() + (ptrdiff_t)i);
        } else {
          i++;
        }
      }
      s->mem_reserved += est;
      s->running++;
      if (large) s->large_running++;
      for (auto &r : batch) s->inflight[r.ticket] = true;
    }
    const Clock::time_point started = Clock::now();
    std::vector<cds::ProblemResult> res;
    cds_status st = CDS_OK;
    std::string msg;
    uint64_t extra = 0;  // reserved after the count
    std::vector<cds_graph *> uploaded;
    // host CSRs are uploaded (and checked) one by one: a malformed one is
    // answered with its own error and leaves the batch
    {
      std::vector<cds_server::Req> ok;
      for (auto &r : batch) {
        if (r.g) {
          ok.push_back(r);
          uploaded.push_back(nullptr);
          continue;
        }
        cds_graph *g = nullptr;
        cds_status ust = CDS_OK;
        std::string umsg;
        try {
          cds::graph_upload(c, stream, r.off, r.adj, r.n, &g);
        } catch (const cds::Error &e) {
          ust = e.status;
          umsg = e.msg;
        }
        if (ust != CDS_OK) {
          std::vector<cds::ProblemResult> none;
          publish(s, {r}, ust, none, started);
          std::lock_guard<std::mutex> g2(c->mu);
          c->err = umsg;
          continue;
        }
        ok.push_back(r);
        uploaded.push_back(g);
      }
      batch.swap(ok);
    }
    if (!batch.empty()) try {
      std::vector<const cds_graph *> gs;
      uint64_t n_all = 0;
      for (size_t i = 0; i < batch.size(); i++) {
        gs.push_back(batch[i].g ? batch[i].g : uploaded[i]);
        n_all += batch[i].n;
      }
      const uint32_t k = batch[0].p.k;
      const cds::CountHook admit = [&](uint64_t cliques) {
        const uint64_t need = post_count_bytes(cliques, k, n_all);
        std::unique_lock<std::mutex> lk(s->mu);
        s->waiting_mem++;
        // wait while it does not fit and some other batch is still working
        // (that one frees memory when it ends); otherwise go ahead, and the
        // allocations themselves decide
        s->cv_mem.wait(lk, [&] {
          return s->mem_reserved + need <= s->budget || s->running == s->waiting_mem || s->stopping;
        });
        s->waiting_mem--;
        s->mem_reserved += need;
        extra += need;
      };
      cds::UnionGraph u;
      cds::build_union(c, stream, gs, u);
      cds::run_problem(c, stream, u, batch[0].p, res, &admit);
    } catch (const cds::Error &e) {
      st = e.status;
      msg = e.msg;
    } catch (const std::exception &e) {
      st = CDS_ERR_STATE;
      msg = e.what();
    }
    for (cds_graph *g : uploaded) {  // freed in this worker's stream order
      if (!g) continue;
      cds::dfree(c, g->d_off, stream);
      cds::dfree(c, g->d_adj, stream);
      delete g;
    }
    if (st != CDS_OK && batch.size() > 1) {
      // split: every request of the batch runs again on its own, first, so
      // a failure (out of memory, or any other) is reported only for the
      // requests that fail alone
      std::lock_guard<std::mutex> lk(s->mu);
      for (auto it = batch.rbegin(); it != batch.rend(); ++it) {
        cds_server::Req r = *it;
        r.alone = true;
        s->inflight.erase(r.ticket);
        s->pending.push_front(r);
      }
    } else if (!batch.empty()) {
      publish(s, batch, st, res, started);
      if (st != CDS_OK) {
        std::lock_guard<std::mutex> g2(c->mu);
        c->err = msg;
      }
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->mem_reserved -= est + extra;
      s->running--;
      if (large) s->large_running--;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    s->cv_mem.notify_all();
  }
}

cds_status enqueue(cds_server *s, cds_server::Req r, uint64_t *ticket) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return CDS_ERR_STATE;
    r.ticket = s->next_ticket++;
    r.submitted = Clock::now();
    s->pending.push_back(r);
    *ticket = r.ticket;
  }
  s->cv_work.notify_all();
  return CDS_OK;
}

}  // namespace

extern "C" {

cds_status cds_server_start(cds_ctx *ctx, const cds_server_config *cfg, cds_server **out) {
  if (!ctx || !out) return CDS_ERR_INPUT;
  cds_server *s = new cds_server();
  s->ctx = ctx;
  if (cfg) s->cfg = *cfg;
  s->budget = s->cfg.mem_budget ? s->cfg.mem_budget : ctx->budget;
  if (s->cfg.max_inflight > CDS_MAX_INFLIGHT) {
    delete s;
    return CDS_ERR_INPUT;
  }
  const size_t nw = s->cfg.max_inflight ? s->cfg.max_inflight
                                        : (ctx->workers.empty() ? 1 : ctx->workers.size());
  s->nworkers = (uint32_t)nw;
  ctx->coop_div.store((int)nw);
  for (size_t i = 0; i < nw; i++) s->workers.emplace_back(worker_main, s, i);
  *out = s;
  return CDS_OK;
}

cds_status cds_submit(cds_server *s, cds_graph *g, const cds_params *params, uint64_t *ticket) {
  if (!s || !g || !params || !ticket) return CDS_ERR_INPUT;
  if (g->ctx != s->ctx) return CDS_ERR_INPUT;
  if (params->k < 2 || params->k > CDS_MAX_K) return CDS_ERR_INPUT;
  cds_server::Req r{};
  r.g = g;
  r.n = g->n;
  r.nnz = g->nnz;
  r.p = *params;
  r.est = pre_count_bytes(g->n, g->nnz, false);
  return enqueue(s, r, ticket);
}

cds_status cds_submit_csr(cds_server *s, const uint64_t *off, const uint32_t *adj, uint32_t n,
                          const cds_params *params, uint64_t *ticket) {
  if (!s || !off || !params || !ticket) return CDS_ERR_INPUT;
  if (params->k < 2 || params->k > CDS_MAX_K) return CDS_ERR_INPUT;
  if (n && off[n] && !adj) return CDS_ERR_INPUT;
  cds_server::Req r{};
  r.off = off;
  r.adj = adj;
  r.n = n;
  r.nnz = off[n];
  r.p = *params;
  r.est = pre_count_bytes(n, r.nnz, true);
  return enqueue(s, r, ticket);
}

static cds_status take(cds_server *s, uint64_t ticket, cds_result *result) {
  auto it = s->done.find(ticket);
  const cds_status st = it->second.st;
  if (st == CDS_OK) {
    try {
      cds::fill_result(it->second.r, result);
    } catch (const cds::Error &e) {
      s->done.erase(it);
      return e.status;
    }
  }
  result->t_queue_ms = it->second.queue_ms;
  result->t_service_ms = it->second.service_ms;
  s->done.erase(it);
  return st;
}

cds_status cds_poll(cds_server *s, uint64_t ticket, cds_result *result) {
  if (!s || !result) return CDS_ERR_INPUT;
  std::memset(result, 0, sizeof(*result));
  std::lock_guard<std::mutex> lk(s->mu);
  if (ticket == 0 || ticket >= s->next_ticket) return CDS_ERR_INPUT;
  if (!s->done.count(ticket)) {
    if (s->inflight.count(ticket)) return CDS_ERR_NOT_READY;
    for (auto &r : s->pending)
      if (r.ticket == ticket) return CDS_ERR_NOT_READY;
    return CDS_ERR_STATE;  // already answered
  }
  return take(s, ticket, result);
}

cds_status cds_wait(cds_server *s, uint64_t ticket, cds_result *result) {
  if (!s || !result) return CDS_ERR_INPUT;
  std::memset(result, 0, sizeof(*result));
  std::unique_lock<std::mutex> lk(s->mu);
  if (ticket == 0 || ticket >= s->next_ticket) return CDS_ERR_INPUT;
  for (;;) {
    if (s->done.count(ticket)) return take(s, ticket, result);
    bool known = s->inflight.count(ticket) > 0;
    for (auto &r : s->pending) known |= r.ticket == ticket;
    if (!known) return CDS_ERR_STATE;  // already answered
    s->cv_done.wait_for(lk, std::chrono::milliseconds(50));
  }
}

cds_status cds_server_stop(cds_server *s) {
  if (!s) return CDS_ERR_INPUT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  s->cv_mem.notify_all();
  for (auto &t : s->workers) t.join();
  s->ctx->coop_div.store(1);
  delete s;
  return CDS_OK;
}

}  // extern "C"
