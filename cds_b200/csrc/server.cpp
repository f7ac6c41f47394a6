// server.cpp -- request loop with continuous batching (cds_server_* in cds.h).
//
// The reference has no serving mode; this is new.  Requests are queued by
// cds_submit.  Up to max_inflight worker threads, one per context stream,
// each take the oldest pending requests that share k (up to max_batch, and
// only while the estimated device memory of the taken requests fits what the
// budget has left), run them as one batched problem, and publish the
// results.  A request that arrives while batches run is admitted by the next
// worker that frees up, so work from different arrivals overlaps on the
// device.  Results are kept until polled.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>

#include "pipeline.h"

struct cds_server {
  cds_ctx *ctx = nullptr;
  cds_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  struct Req {
    uint64_t ticket;
    cds_graph *g;
    cds_params p;
    uint64_t est;
  };
  std::deque<Req> pending;
  struct Done {
    cds_status st;
    cds::ProblemResult r;
  };
  std::map<uint64_t, Done> done;
  std::map<uint64_t, bool> inflight;  // tickets a worker is solving
  uint64_t next_ticket = 1;
  uint64_t mem_reserved = 0;
  uint64_t budget = 0;
  uint32_t running = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
};

namespace {

// Device bytes one request may need: its graph's DAG and work arrays, plus
// the clique store and flow state bounded through the partition sizes the
// request carries (pSize/cpSize listing partitions, partitionSize flow
// queue), as the reference sizes its buffers from the same arguments.
uint64_t estimate(const cds_graph *g, const cds_params &p) {
  const uint64_t n = g->n, nnz = g->nnz;
  uint64_t b = 64 * (n + 1) + 8 * nnz;
  const uint64_t part = (uint64_t)p.p_size + p.cp_size;
  b += 16 * part * (p.k ? p.k : 1);
  b += 48 * (uint64_t)p.partition_size;
  return b + (1u << 20);
}

void worker_main(cds_server *s, size_t wi) {
  cds_ctx *c = s->ctx;
  cudaStream_t stream = c->workers.empty() ? c->stream : c->workers[wi % c->workers.size()];
  cudaSetDevice(c->device);
  for (;;) {
    std::vector<cds_server::Req> batch;
    uint64_t est = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stopping || !s->pending.empty(); });
      if (s->pending.empty()) {
        if (s->stopping) return;
        continue;
      }
      const uint32_t k = s->pending.front().p.k;
      const uint32_t cap = s->cfg.max_batch ? s->cfg.max_batch : 64;
      for (auto it = s->pending.begin(); it != s->pending.end() && batch.size() < cap;) {
        if (it->p.k == k && it->p.search == s->pending.front().p.search &&
            it->p.early_stop == s->pending.front().p.early_stop &&
            (batch.empty() || s->mem_reserved + est + it->est <= s->budget)) {
          est += it->est;
          batch.push_back(*it);
          it = s->pending.erase(it);
        } else {
          ++it;
        }
      }
      s->mem_reserved += est;
      s->running++;
      for (auto &r : batch) s->inflight[r.ticket] = true;
    }
    std::vector<cds::ProblemResult> res;
    cds_status st = CDS_OK;
    std::string msg;
    try {
      std::vector<const cds_graph *> gs;
      for (auto &r : batch) gs.push_back(r.g);
      cds::UnionGraph u;
      cds::build_union(c, stream, gs, u);
      cds::run_problem(c, stream, u, batch[0].p, res);
    } catch (const cds::Error &e) {
      st = e.status;
      msg = e.msg;
    } catch (const std::exception &e) {
      st = CDS_ERR_STATE;
      msg = e.what();
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (size_t i = 0; i < batch.size(); i++) {
        cds_server::Done d;
        d.st = st;
        if (st == CDS_OK) d.r = std::move(res[i]);
        s->done[batch[i].ticket] = std::move(d);
        s->inflight.erase(batch[i].ticket);
      }
      if (st != CDS_OK) {
        std::lock_guard<std::mutex> g2(c->mu);
        c->err = msg;
      }
      s->mem_reserved -= est;
      s->running--;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
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
  ctx->coop_div.store((int)nw);
  for (size_t i = 0; i < nw; i++) s->workers.emplace_back(worker_main, s, i);
  *out = s;
  return CDS_OK;
}

cds_status cds_submit(cds_server *s, cds_graph *g, const cds_params *params, uint64_t *ticket) {
  if (!s || !g || !params || !ticket) return CDS_ERR_INPUT;
  if (g->ctx != s->ctx) return CDS_ERR_INPUT;
  if (params->k < 2 || params->k > CDS_MAX_K) return CDS_ERR_INPUT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return CDS_ERR_STATE;
    const uint64_t t = s->next_ticket++;
    s->pending.push_back({t, g, *params, estimate(g, *params)});
    *ticket = t;
  }
  s->cv_work.notify_one();
  return CDS_OK;
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
  for (auto &t : s->workers) t.join();
  s->ctx->coop_div.store(1);
  delete s;
  return CDS_OK;
}

}  // extern "C"
