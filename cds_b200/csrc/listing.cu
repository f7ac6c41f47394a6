// listing.cu -- k-clique counting and listing.
//
// Replaces listAllCliques (cudaCode/main.cu:59-250) and its kernels
// listIntialCliques / flushParitions / listMidCliques / countCliques /
// writeFinalCliques (cudaCode/src/helpers.cu:175-574, 1098-1137), and the
// k = 2 path writeEdgeCliques (helpers.cu:576-609).
//
// Every vertex u with out-degree d >= k-1 is a root.  A team (one warp for
// d <= 128, one block above that) stages N+(u) = A[0..d) in shared memory
// with 128-bit loads and builds the local adjacency bitmap: bit j of row i
// is set when A[j] is an out-neighbour of A[i] (each lane binary-searches one
// element of N+(A[i]) in A).  The k-cliques rooted at u are then
// u, A[i], A[j] plus a (k-3)-clique inside row_i & row_j, found with AND and
// popcount on the bitmaps.  The (i, j) pairs (the set bits of all rows) are
// numbered 0..P-1 through a prefix over row popcounts, and the team's threads
// take consecutive pair numbers, so work is balanced inside a root whatever
// the row lengths.
//
// Pass 1 (count) sums the cliques of each root and accumulates each vertex's
// clique degree in shared memory before one atomic per vertex and root.
// Pass 2 (write) re-enumerates and stores clique records (k ids) at the
// root's offset from the prefix of pass-1 counts, so the record order is the
// root order: deterministic, independent of scheduling.
#include "device_util.cuh"
#include "stages.h"

#include "list_kernels.cuh"

namespace {

// k = 2: every DAG arc is a clique
__global__ void k_edges_write(const uint64_t *__restrict__ doff, const uint32_t *__restrict__ dadj,
                              const uint32_t *__restrict__ outdeg, const uint64_t *__restrict__ base,
                              uint32_t n, uint32_t *__restrict__ out) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint32_t d = outdeg[v];
    const uint64_t b = base[v];
    for (uint32_t t = lane_id(); t < d; t += 32)
      *reinterpret_cast<uint2 *>(out + (b + t) * 2) = make_uint2(v, dadj[doff[v] + t]);
  }
}

__global__ void k_copy_u32(const uint32_t *a, uint32_t *b, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    b[v] = a[v];
}

__global__ void k_widen(const uint32_t *a, unsigned long long *b, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    b[v] = a[v];
}

// u32 copy of the clique degrees; err |= DEV_ERR_OVERFLOW for one >= 2^32
__global__ void k_narrow(const unsigned long long *a, uint32_t *b, uint32_t n, uint32_t *err) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const unsigned long long x = a[v];
    if (x > 0xFFFFFFFFull) atomicOr(err, DEV_ERR_OVERFLOW);
    b[v] = (uint32_t)x;
  }
}

template <int K>
void launch_pass(cds_ctx *c, cudaStream_t s, const cds::Tuning &t, ListParams p, bool write,
                 bool block_team, uint32_t grid_cap) {
  const int threads = block_team ? t.list_team_block : t.list_warp_block;
  size_t smem;
  if (block_team) {
    smem = (size_t)p.team_words * 4;
  } else {
    smem = (size_t)p.team_words * 4 * (threads / 32);
  }
  void (*fn)(ListParams);
  if (block_team) fn = write ? k_list<K, true, true> : k_list<K, false, true>;
  else fn = write ? k_list<K, true, false> : k_list<K, false, false>;
  // The limit is a property of the kernel shared by every thread of the
  // process: concurrent solves (server workers) launch it with different
  // sizes, so it is raised to the device's maximum rather than set to this
  // launch's size, which another thread could lower before this launch.
  cudaFuncAttributes fa;
  CDS_CUDA(cudaFuncGetAttributes(&fa, fn));
  const size_t dyn_max = c->smem_optin - fa.sharedSizeBytes;  // the rest is the kernel's static use
  if (smem > dyn_max) cds::fail(CDS_ERR_CUDA, "listing team does not fit in shared memory");
  CDS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_max));
  int per_sm = 0;
  CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  if (per_sm < 1) cds::fail(CDS_ERR_CUDA, "listing kernel does not fit on an SM");
  uint32_t grid = (uint32_t)(c->sm_count * per_sm);
  if (grid_cap && grid > grid_cap) grid = grid_cap;
  static const char *names[2][2] = {{"list_count_warp", "list_count_block"},
                                    {"list_write_warp", "list_write_block"}};
  cds::ProfScope ps(c, s, names[write ? 1 : 0][block_team ? 1 : 0]);
  fn<<<grid, threads, smem, s>>>(p);
  cds::count_launch();
  CDS_CUDA(cudaGetLastError());
}

template <int K>
void run_listing(cds_ctx *c, cudaStream_t s, const cds::Dag &dag, bool materialize,
                 const cds::Tuning &t, cds::Cliques &out, uint32_t *err, uint32_t k,
                 const cds::CountHook *on_count) {
  using namespace cds;
  const uint32_t n = dag.n;
  const uint32_t warp_dmax = (uint32_t)std::min(t.list_warp_dmax, WARP_DMAX);
  DBuf<uint32_t> lists(c, s, 2 * (size_t)n + 2);
  DBuf<uint32_t> counters(c, s, 8);
  counters.zero();
  uint32_t *wl = lists.p, *bl = lists.p + n + 1;
  k_classify<<<c->sm_count * 4, 256, 0, s>>>(dag.outdeg.p, n, k - 1, warp_dmax, wl,
                                             counters.p, bl, counters.p + 1);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  // the root counts stay on the device (the kernels read them), so nothing
  // waits here; a pass whose team kind has no roots exits at once

  DBuf<unsigned long long> root_cnt(c, s, n + 1);
  root_cnt.zero();
  out.cdeg64.zero();

  ListParams p{};
  p.doff = dag.off.p;
  p.dadj = dag.adj.p;
  p.outdeg = dag.outdeg.p;
  p.cdeg = nullptr;
  p.cdeg64 = out.cdeg64.p;
  p.root_cnt = root_cnt.p;
  p.err = err;
  p.k = k;

  // block-team geometry
  const uint32_t bdmax = std::max<uint32_t>(dag.max_out, warp_dmax + 1);
  const bool rows_in_smem = bdmax <= (uint32_t)BLOCK_DMAX;
  const uint32_t bw = (bdmax + 31) / 32;
  const uint64_t brow_words = (uint64_t)bdmax * (bw | 1u);
  DBuf<uint32_t> rows_global;
  uint32_t bgrid_cap = 0;
  const bool any_block = dag.max_out > warp_dmax;
  if (any_block && !rows_in_smem) {
    bgrid_cap = (uint32_t)c->sm_count;
    rows_global.alloc((size_t)bgrid_cap * brow_words);
  }

  auto pass = [&](bool write) {
    {
      ListParams q = p;
      q.roots = wl;
      q.nroots = counters.p;
      q.work = counters.p + 2 + (write ? 1 : 0);
      q.dmax = warp_dmax;
      q.team_words = warp_dmax + (warp_dmax + 1) + warp_dmax + warp_dmax * (((warp_dmax + 31) / 32) | 1u);
      q.team_words = (q.team_words + 3) & ~3u;
      launch_pass<K>(c, s, t, q, write, false, 0);
    }
    if (any_block) {
      ListParams q = p;
      q.roots = bl;
      q.nroots = counters.p + 1;
      q.work = counters.p + 4 + (write ? 1 : 0);
      q.dmax = bdmax;
      q.team_words = bdmax + (bdmax + 1) + bdmax + (rows_in_smem ? (uint32_t)brow_words : 0u);
      q.team_words = (q.team_words + 3) & ~3u;
      q.rows_global = rows_in_smem ? nullptr : rows_global.p;
      q.rows_slab = brow_words;
      launch_pass<K>(c, s, t, q, write, true, bgrid_cap);
    }
  };
  pass(false);
  out.base.alloc(n + 1);
  scan_u64(reinterpret_cast<const uint64_t *>(root_cnt.p), out.base.p, n, c, s);
  out.count = d2h(out.base.p + n, s);
  if (on_count) (*on_count)(out.count);
  if (!materialize) return;
  // later stages keep clique degrees (and core numbers) as u32
  if (n) {
    k_narrow<<<c->sm_count * 4, 256, 0, s>>>(out.cdeg64.p, out.cdeg.p, n, err);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
  out.members.alloc((size_t)out.count * k + 4);
  p.base = reinterpret_cast<const unsigned long long *>(out.base.p);
  p.out = out.members.p;
  pass(true);
}

}  // namespace

namespace cds {

void list_cliques(cds_ctx *c, cudaStream_t s, const Dag &dag, uint32_t k, bool materialize,
                  const Tuning &t, Cliques &out, const CountHook *on_count) {
  if (k < 2 || k > CDS_MAX_K) fail(CDS_ERR_INPUT, "k must be in [2, 16]");
  const uint32_t n = dag.n;
  out.k = k;
  out.cdeg.c = c;
  out.cdeg.s = s;
  out.cdeg64.c = c;
  out.cdeg64.s = s;
  out.base.c = c;
  out.base.s = s;
  out.members.c = c;
  out.members.s = s;
  out.cdeg64.alloc(n + 1);
  if (materialize) out.cdeg.alloc(n + 1);
  DBuf<uint32_t> err(c, s, 1);
  err.zero();
  if (k == 2) {
    // every edge is a 2-clique; the clique degree is the degree
    out.base.alloc(n + 1);
    scan_u32(dag.outdeg.p, out.base.p, n, c, s);
    out.count = d2h(out.base.p + n, s);
    if (on_count) (*on_count)(out.count);
    if (n) {
      k_widen<<<c->sm_count * 4, 256, 0, s>>>(dag.deg.p, out.cdeg64.p, n);
      if (materialize) k_copy_u32<<<c->sm_count * 4, 256, 0, s>>>(dag.deg.p, out.cdeg.p, n);
      count_launch(materialize ? 2 : 1);
    }
    if (materialize) {
      out.members.alloc((size_t)out.count * 2 + 4);
      if (n) {
        ProfScope ps(c, s, "list_write_edges");
        k_edges_write<<<c->sm_count * 8, 256, 0, s>>>(dag.off.p, dag.adj.p, dag.outdeg.p,
                                                       out.base.p, n, out.members.p);
        count_launch();
      }
    }
    CDS_CUDA(cudaGetLastError());
    return;
  }
  if (k == 3) run_listing<3>(c, s, dag, materialize, t, out, err.p, k, on_count);
  else if (k == 4) run_listing<4>(c, s, dag, materialize, t, out, err.p, k, on_count);
  else run_listing<0>(c, s, dag, materialize, t, out, err.p, k, on_count);
  const uint32_t e = d2h(err.p, s);
  if (e & DEV_ERR_OVERFLOW)
    fail(CDS_ERR_OVERFLOW, "a root's out-degree exceeds the k >= 5 listing's masks, or a clique degree "
                           "reaches 2^32 (the later stages keep clique degrees as u32)");
  if (e) fail(CDS_ERR_CUDA, "listing kernel reported an internal error");
}

}  // namespace cds
