// noalloc.cu -- cds_count_cliques_noalloc: the k-clique count and clique
// degrees of a device-resident graph, written into buffers the caller owns,
// with no device allocation at all.
//
// Who needs it: code running under a framework or memory manager that owns
// every device allocation of the process (a caching allocator that has
// reserved the device up front, an embedding host with a fixed device
// budget) cannot call cudaMalloc, or anything that allocates, in the middle
// of its work: the call would fail for lack of memory, or take memory the
// owner has already promised elsewhere.  This entry point keeps every scratch
// array it needs in one file-scope __device__ array, g_scratch below, sized
// for the limits NA_MAX_* (about 21 MiB; every GPU that loads libcds holds it
// until the process exits).  The caller still allocates its inputs and
// outputs.
//
// The call checks its input and reads a few scalars back, each with a wait on
// the caller's stream, and returns once the count is complete.
//
// It runs the same DAG and listing kernels as cds_list_cliques
// (dag_kernels.cuh, list_kernels.cuh), with the scan and the small helpers
// below working on slices of g_scratch.
#include <cstring>
#include <mutex>

#include "cds_internal.h"
#include "dag_kernels.cuh"
#include "list_kernels.cuh"

namespace {

constexpr uint32_t NA_MAX_N = 1u << 18;       // vertices
constexpr uint64_t NA_MAX_ARCS = 1ull << 22;  // directed arcs, off[n] (m <= 2^21 edges)
constexpr uint32_t NA_MAX_OUT = 1024;         // DAG out-degree (bitmap rows in shared memory)
constexpr uint32_t NA_WARP_DMAX = 128;
constexpr int NA_MAX_DEVICES = 64;

constexpr size_t al(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t NA_TILES = (NA_MAX_N + SCAN_TILE) / SCAN_TILE;
// scratch layout, byte offsets of 256-byte aligned regions
constexpr size_t S_DEG = 0;                                         // u32 [n+1]
constexpr size_t S_OUTDEG = S_DEG + al(4 * (NA_MAX_N + 1));         // u32 [n+1]
constexpr size_t S_DOFF = S_OUTDEG + al(4 * (NA_MAX_N + 1));        // u64 [n+1]
constexpr size_t S_DADJ = S_DOFF + al(8 * (NA_MAX_N + 1));          // u32 [m + 3n + 4]
constexpr size_t S_RCNT = S_DADJ + al(4 * (NA_MAX_ARCS / 2 + 3 * (size_t)NA_MAX_N + 4));  // u64 [n+1]
constexpr size_t S_LIST = S_RCNT + al(8 * (NA_MAX_N + 1));          // u32 [2(n+1)]
constexpr size_t S_TSUM = S_LIST + al(8 * (NA_MAX_N + 1));          // u64 [tiles]
constexpr size_t S_TOFF = S_TSUM + al(8 * NA_TILES);                // u64 [tiles+1]
constexpr size_t S_CDEG = S_TOFF + al(8 * (NA_TILES + 1));          // u32 [n+1]
constexpr size_t S_CTL = S_CDEG + al(4 * (NA_MAX_N + 1));           // u32 [64]
constexpr size_t NA_BYTES = S_CTL + 256;
enum { C_BAD = 0, C_MAXOUT = 1, C_NW = 2, C_NB = 3, C_WORK = 4, C_ERR = 8 };

__device__ __align__(256) unsigned char g_scratch[NA_BYTES];

std::mutex g_mu;
unsigned char *g_base[NA_MAX_DEVICES];  // device address of g_scratch, per device

// First check, on the offsets alone: off[0] = 0 and off[v] <= off[v+1] for
// every v < n, so every row lies inside [0, off[n]), the arcs the caller's
// adjacency array holds.  Nothing here reads the adjacency array.
__global__ void k_na_check_off(const uint64_t *__restrict__ off, uint32_t n, uint32_t *__restrict__ bad) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (off[v] > off[v + 1] || (v == 0 && off[0] != 0)) atomicOr(bad, 1u);
}

// Second check, run only once the offsets passed: rows strictly ascending,
// no self-loops, ids < n, every arc has its reverse.  An id is compared with
// n before it indexes anything.
__global__ void k_na_check(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                           uint32_t n, uint32_t *__restrict__ bad) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = off[v], e = off[v + 1];
    uint32_t flag = e < b;
    for (uint64_t i = b + lane_id(); i < e && !flag; i += 32) {
      const uint32_t w = adj[i];
      if (w >= n || w == v || (i > b && adj[i - 1] >= w)) {
        flag = 1;
        break;
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

// exclusive scan of the padded out-degrees: tiles, tile sums (one block), add
__global__ void __launch_bounds__(SCAN_THREADS) k_na_scan_tiles(const uint32_t *in, uint64_t *out,
                                                                uint64_t *sums, uint32_t n) {
  const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS];
  uint64_t t = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = base + i < n ? (uint64_t)((in[base + i] + 3u) & ~3u) : 0;
    t += v[i];
  }
  uint64_t total;
  uint64_t ex = block_exclusive_scan<uint64_t>(t, &total);
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) out[base + i] = ex;
    ex += v[i];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void k_na_scan_sums(const uint64_t *sums, uint64_t *toff, uint32_t tiles) {
  // tiles <= 128 = blockDim.x
  const uint64_t x = threadIdx.x < tiles ? sums[threadIdx.x] : 0;
  uint64_t total;
  const uint64_t ex = block_exclusive_scan<uint64_t>(x, &total);
  if (threadIdx.x < tiles) toff[threadIdx.x] = ex;
  if (threadIdx.x == 0) toff[tiles] = total;
}
__global__ void k_na_scan_add(uint64_t *out, const uint64_t *toff, uint32_t n, uint32_t tiles) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += toff[i / SCAN_TILE];
  if (i == 0) out[n] = toff[tiles];
}

__global__ void k_na_copy(const uint32_t *a, uint32_t *b, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    b[v] = a[v];
}

__global__ void k_na_set(unsigned long long *dst, unsigned long long v) { *dst = v; }

__global__ void k_na_sum(const unsigned long long *a, uint32_t n, unsigned long long *out) {
  unsigned long long t = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    t += a[v];
  t = warp_sum(t);
  if (lane_id() == 0 && t) atomicAdd(out, t);
}

template <int K>
cds_status launch_count(ListParams p, bool block_team, int sms, cudaStream_t s) {
  const int threads = block_team ? 512 : 256;
  const size_t smem = block_team ? (size_t)p.team_words * 4 : (size_t)p.team_words * 4 * (threads / 32);
  void (*fn)(ListParams) = block_team ? k_list<K, false, true> : k_list<K, false, false>;
  // raised to the device maximum, never lowered: the listing kernels are
  // shared with the allocating entry points, which may run in other threads
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, fn) != cudaSuccess)
    return CDS_ERR_CUDA;
  const size_t dyn_max = (size_t)optin - fa.sharedSizeBytes;  // the rest is the kernel's static use
  if (dyn_max < smem) return CDS_ERR_CUDA;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_max) != cudaSuccess)
    return CDS_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1)
    return CDS_ERR_CUDA;
  fn<<<sms * per_sm, threads, smem, s>>>(p);
  cds::count_launch();
  return cudaGetLastError() == cudaSuccess ? CDS_OK : CDS_ERR_CUDA;
}

template <int K>
cds_status count_pass(ListParams p, uint32_t nw, uint32_t nb, const uint32_t *d_nw, const uint32_t *d_nb,
                      uint32_t bdmax, uint32_t *wl, uint32_t *bl, uint32_t *work, int sms,
                      cudaStream_t s) {
  cds_status st = CDS_OK;
  if (nw) {
    ListParams q = p;
    q.roots = wl;
    q.nroots = d_nw;
    q.work = work;
    q.dmax = NA_WARP_DMAX;
    q.team_words = (NA_WARP_DMAX + (NA_WARP_DMAX + 1) + NA_WARP_DMAX +
                    NA_WARP_DMAX * (((NA_WARP_DMAX + 31) / 32) | 1u) + 3) & ~3u;
    st = launch_count<K>(q, false, sms, s);
    if (st != CDS_OK) return st;
  }
  if (nb) {
    ListParams q = p;
    q.roots = bl;
    q.nroots = d_nb;
    q.work = work + 1;
    q.dmax = bdmax;
    q.team_words = (bdmax + (bdmax + 1) + bdmax + bdmax * (((bdmax + 31) / 32) | 1u) + 3) & ~3u;
    q.rows_global = nullptr;
    st = launch_count<K>(q, true, sms, s);
  }
  return st;
}

#define NA_TRY(call)                                   \
  do {                                                 \
    if ((call) != cudaSuccess) return CDS_ERR_CUDA;    \
  } while (0)

}  // namespace

extern "C" cds_status cds_count_cliques_noalloc(const uint64_t *d_off, const uint32_t *d_adj,
                                                uint32_t n, uint32_t k,
                                                unsigned long long *d_count,
                                                uint32_t *d_clique_degree, void *stream) {
  if (!d_off || !d_count || k < 2 || k > CDS_MAX_K) return CDS_ERR_INPUT;
  if (n > NA_MAX_N) return CDS_ERR_INPUT;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  NA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return CDS_ERR_INPUT;
  NA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  unsigned char *base = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_base[dev]) {
      void *ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || !ptr) return CDS_ERR_CUDA;
      g_base[dev] = (unsigned char *)ptr;
    }
    base = g_base[dev];
  }
  uint32_t *deg = (uint32_t *)(base + S_DEG);
  uint32_t *outdeg = (uint32_t *)(base + S_OUTDEG);
  uint64_t *doff = (uint64_t *)(base + S_DOFF);
  uint32_t *dadj = (uint32_t *)(base + S_DADJ);
  unsigned long long *rcnt = (unsigned long long *)(base + S_RCNT);
  uint32_t *wl = (uint32_t *)(base + S_LIST);
  uint32_t *bl = wl + NA_MAX_N + 1;
  uint64_t *tsum = (uint64_t *)(base + S_TSUM);
  uint64_t *toff = (uint64_t *)(base + S_TOFF);
  uint32_t *cdeg = d_clique_degree ? d_clique_degree : (uint32_t *)(base + S_CDEG);
  uint32_t *ctl = (uint32_t *)(base + S_CTL);

  // The scratch keeps the last call's contents: clear what counts from zero.
  // The input is checked in two steps, each read back before anything uses
  // it as an index: first the offsets (with the arc count), then the ids.
  NA_TRY(cudaMemsetAsync(ctl, 0, 256, s));
  NA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s));
  const int grid = sms * 8;
  if (n) {
    k_na_check_off<<<grid, 256, 0, s>>>(d_off, n, ctl + C_BAD);
    cds::count_launch();
    NA_TRY(cudaGetLastError());
  }
  uint64_t nnz = 0;
  uint32_t bad = 0;
  NA_TRY(cudaMemcpyAsync(&nnz, d_off + n, sizeof(nnz), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaMemcpyAsync(&bad, ctl + C_BAD, sizeof(bad), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaStreamSynchronize(s));
  if (bad) return CDS_ERR_INPUT;  // offsets not starting at 0 or decreasing
  if (nnz > NA_MAX_ARCS || (nnz && !d_adj)) return CDS_ERR_INPUT;
  if (n == 0) return nnz ? CDS_ERR_INPUT : CDS_OK;
  k_na_check<<<grid, 256, 0, s>>>(d_off, d_adj, n, ctl + C_BAD);
  cds::count_launch();
  NA_TRY(cudaGetLastError());
  NA_TRY(cudaMemcpyAsync(&bad, ctl + C_BAD, sizeof(bad), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaStreamSynchronize(s));
  if (bad) return CDS_ERR_INPUT;  // not a symmetric CSR with ascending rows
  NA_TRY(cudaMemsetAsync(rcnt, 0, 8 * ((size_t)n + 1), s));
  NA_TRY(cudaMemsetAsync(cdeg, 0, 4 * (size_t)n, s));

  k_degree<<<grid, 256, 0, s>>>(d_off, n, deg);
  k_outdeg<<<grid, 256, 0, s>>>(d_off, d_adj, deg, n, outdeg, ctl + C_MAXOUT);
  const uint32_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  k_na_scan_tiles<<<tiles, SCAN_THREADS, 0, s>>>(outdeg, doff, tsum, n);
  k_na_scan_sums<<<1, 128, 0, s>>>(tsum, toff, tiles);
  k_na_scan_add<<<(n + 255) / 256, 256, 0, s>>>(doff, toff, n, tiles);
  cds::count_launch(5);
  NA_TRY(cudaGetLastError());
  uint32_t hctl[2] = {0, 0};
  uint64_t dag_arcs = 0;
  NA_TRY(cudaMemcpyAsync(hctl, ctl, sizeof(hctl), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaMemcpyAsync(&dag_arcs, doff + n, sizeof(dag_arcs), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaStreamSynchronize(s));
  if (hctl[C_MAXOUT] > NA_MAX_OUT) return CDS_ERR_INPUT;
  if (dag_arcs > NA_MAX_ARCS / 2 + 3 * (uint64_t)NA_MAX_N + 4) return CDS_ERR_INPUT;
  k_dag_fill<<<grid, 256, 0, s>>>(d_off, d_adj, deg, n, doff, dadj);
  cds::count_launch();
  NA_TRY(cudaGetLastError());
  if (k == 2) {  // every edge is a 2-clique
    k_na_copy<<<grid, 256, 0, s>>>(deg, cdeg, n);
    k_na_set<<<1, 1, 0, s>>>(d_count, nnz / 2);
    cds::count_launch(2);
    return cudaGetLastError() == cudaSuccess ? CDS_OK : CDS_ERR_CUDA;
  }
  k_classify<<<sms * 4, 256, 0, s>>>(outdeg, n, k - 1, NA_WARP_DMAX, wl, ctl + C_NW, bl, ctl + C_NB);
  cds::count_launch();
  uint32_t hn[2] = {0, 0};
  NA_TRY(cudaMemcpyAsync(hn, ctl + C_NW, sizeof(hn), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaStreamSynchronize(s));
  ListParams p{};
  p.doff = doff;
  p.dadj = dadj;
  p.outdeg = outdeg;
  p.cdeg = cdeg;
  p.root_cnt = rcnt;
  p.err = ctl + C_ERR;
  p.k = k;
  const uint32_t bdmax = hctl[C_MAXOUT] > NA_WARP_DMAX ? hctl[C_MAXOUT] : NA_WARP_DMAX + 1;
  cds_status st;
  if (k == 3) st = count_pass<3>(p, hn[0], hn[1], ctl + C_NW, ctl + C_NB, bdmax, wl, bl, ctl + C_WORK, sms, s);
  else if (k == 4) st = count_pass<4>(p, hn[0], hn[1], ctl + C_NW, ctl + C_NB, bdmax, wl, bl, ctl + C_WORK, sms, s);
  else st = count_pass<0>(p, hn[0], hn[1], ctl + C_NW, ctl + C_NB, bdmax, wl, bl, ctl + C_WORK, sms, s);
  if (st != CDS_OK) return st;
  k_na_sum<<<sms, 256, 0, s>>>(rcnt, n, d_count);
  cds::count_launch();
  NA_TRY(cudaGetLastError());
  // the listing kernels flag a root they could not enumerate (out-degree
  // above the team's rows, or a clique deeper than their masks): the count
  // would be short, so the call fails instead
  uint32_t lerr = 0;
  NA_TRY(cudaMemcpyAsync(&lerr, ctl + C_ERR, sizeof(lerr), cudaMemcpyDeviceToHost, s));
  NA_TRY(cudaStreamSynchronize(s));
  if (lerr & DEV_ERR_OVERFLOW) return CDS_ERR_OVERFLOW;
  return lerr ? CDS_ERR_CUDA : CDS_OK;
}
