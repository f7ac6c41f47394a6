// cds_internal.h -- host-side state behind the C ABI: context, graphs,
// device buffers and the per-stage launch interfaces.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "cds.h"

namespace cds {

// Internal failures travel as exceptions and become a cds_status at the ABI.
struct Error {
  cds_status status;
  std::string msg;
};
[[noreturn]] void fail(cds_status s, const std::string &msg);
void cuda_check(cudaError_t e, const char *what);
#define CDS_CUDA(call) ::cds::cuda_check((call), #call)

// Launch shapes chosen by the autotuner (per clique size).
struct Tuning {
  int list_warp_block = 256;   // threads per block, warp-per-root listing
  int list_team_block = 512;   // threads per block, block-per-root listing
  int list_warp_dmax = 128;    // largest out-degree handled by one warp
  int flow_block = 512;        // threads per block, push-relabel
  int flow_rounds = 16;        // push/relabel rounds between global relabels
  int flow_warm = -1;          // balancing rounds before each max-flow (0: none;
                               // < 0: three for networks of 2^20 cliques or more)
  int flow_inc_per_block = 0;  // push-relabel grid: a block per this many incidences
                               // (0: the whole device); small networks then
                               // meet at cheaper grid barriers
  int peel_chunk = 512;        // incidences per peel work item
  int peel_order = 0;          // peel items by ascending clique-degree class (1) or vertex id (0)
  int peel_static = 100;       // percent of peel items dealt round-robin; the rest by a counter
};

}  // namespace cds

namespace cds {
struct ProfEvent {
  const char *name;
  cudaEvent_t a, b;
};
}  // namespace cds

struct cds_ctx {
  int device = 0;
  uint32_t flags = 0;  // CDS_CONFIG_* bits
  int sm_count = 0;
  size_t smem_optin = 0;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> workers;
  cudaMemPool_t pool = nullptr;
  uint64_t budget = 0;
  std::atomic<uint64_t> in_use{0};
  std::atomic<uint64_t> peak{0};
  std::mutex mu;  // guards sizes and err
  std::unordered_map<void *, size_t> sizes;
  std::string err;
  cds::Tuning tune[CDS_MAX_K + 1];
  // Cooperative (grid-barrier) kernels use 1/coop_div of the device, so that
  // coop_div of them launched from concurrent server workers can all be
  // resident at once; 1 outside serving.
  std::atomic<int> coop_div{1};
  // kernel profiling (cds_profile): events resolved at cds_profile_read
  bool prof = false;
  std::vector<cds::ProfEvent> prof_pending;
  std::unordered_map<std::string, std::pair<uint64_t, double>> prof_done;
};

struct cds_graph {
  cds_ctx *ctx = nullptr;
  uint32_t n = 0;
  uint64_t nnz = 0;  // directed arcs = 2m
  uint32_t max_degree = 0;
  uint64_t *d_off = nullptr;  // [n+1]
  uint32_t *d_adj = nullptr;  // [nnz]
  std::vector<uint64_t> h_off;
  std::vector<uint32_t> h_adj;
};

namespace cds {

// Stream-ordered device allocation against the context budget.
void *dalloc_bytes(cds_ctx *c, size_t bytes, cudaStream_t s);
void dfree(cds_ctx *c, void *p, cudaStream_t s);

template <class T>
struct DBuf {
  cds_ctx *c = nullptr;
  cudaStream_t s = nullptr;
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(cds_ctx *c_, cudaStream_t s_, size_t n_) : c(c_), s(s_) { alloc(n_); }
  void alloc(size_t n_) {
    release();
    n = n_;
    p = n ? (T *)dalloc_bytes(c, n * sizeof(T), s) : nullptr;
  }
  void zero() {
    if (n) CDS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void release() {
    if (p) dfree(c, p, s);
    p = nullptr;
    n = 0;
  }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : c(o.c), s(o.s), p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    release();
    c = o.c; s = o.s; p = o.p; n = o.n;
    o.p = nullptr; o.n = 0;
    return *this;
  }
  ~DBuf() { release(); }
};

// exclusive scan: out[0..n] with out[n] = total
void scan_u32(const uint32_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s);
void scan_u64(const uint64_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s);
// exclusive scan of (in[i] + 3) & ~3 (rows padded to 16 bytes)
void scan_u32_pad4(const uint32_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s);

// Device-to-host reads of a stage's small results.  A copy into pageable
// host memory returns only once it has completed, so every such copy is a
// full wait on the stream; these go through a pinned buffer of the calling
// thread (1 MiB, allocated on first use) instead, and a group of them costs
// one wait.  add() queues a copy; wait() waits once and moves the values to
// their destinations.  Groups take space from the thread's buffer like a
// stack (a group opened inside another finishes first); a read that does not
// fit is copied directly at wait().
class HostReads {
 public:
  explicit HostReads(cudaStream_t s);
  ~HostReads();
  HostReads(const HostReads &) = delete;
  HostReads &operator=(const HostReads &) = delete;
  template <class T>
  void add(T *dst, const T *src, size_t count = 1) { add_bytes(dst, src, count * sizeof(T)); }
  void add_bytes(void *dst, const void *src, size_t bytes);
  void wait();

 private:
  struct Item {
    void *dst;
    const void *src;
    size_t off, bytes;  // off = SIZE_MAX: read directly
  };
  cudaStream_t s_;
  size_t base_;
  std::vector<Item> items_;
};

template <class T>
T d2h(const T *d, cudaStream_t s) {
  T h;
  HostReads r(s);
  r.add(&h, d);
  r.wait();
  return h;
}

// Device-event timing of one kernel launch when profiling is on.
struct ProfScope {
  cds_ctx *c;
  cudaStream_t s;
  const char *name;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(cds_ctx *c_, cudaStream_t s_, const char *name_) : c(c_), s(s_), name(name_) {
    if (!c->prof) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  ~ProfScope() {
    if (!a) return;
    cudaEventRecord(b, s);
    std::lock_guard<std::mutex> g(c->mu);
    c->prof_pending.push_back({name, a, b});
  }
};

// Counts every kernel launch made by the library (for reporting).
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Blocks of a cooperative launch: per_sm blocks on every SM, divided among
// the cooperative kernels that may run concurrently.
inline unsigned coop_grid(const cds_ctx *c, int per_sm) {
  const int d = c->coop_div.load();
  const int g = c->sm_count * per_sm / (d > 0 ? d : 1);
  return (unsigned)(g > 0 ? g : 1);
}

}  // namespace cds

extern "C" uint64_t cds_kernel_launches(void);
