// parse.cu -- adjacency-list text and binary CSR files into a canonical
// device CSR, parsed on the device.
//
// Replaces the host readers Graph::Graph (cudaCode/src/graph.cpp:7-40) and
// cpuCode/c++/src/graph.cpp:9-52, which read the file line by line with
// string streams on one host thread.  Here the host reads the bytes once and
// every later step runs on the device:
//   1. token boundaries: a byte starts a token when it is a digit and the
//      byte before is not; a token ends a line when the next separator run
//      holds a newline.  Both are flags per byte, compacted by a scan into
//      token start positions and a line index per token.
//   2. values: one thread per token reads its digits (at most 10).
//   3. the header line gives n; on every later line the first token is the
//      vertex v and the others its neighbours w: each (v, w) with w != v is
//      counted for both endpoints, scattered into rows, and each row is
//      sorted and de-duplicated (symmetric, ascending, no self-loops --
//      the same canonical CSR as the host reader cds_read_adjlist).
// Rows are sorted by one block each: bitonic in shared memory up to
// SMEM_SORT entries, in global memory (the row's own slice, padded) above.
//
// The binary CSR cache (cds_csr_write_binary) skips the text entirely: a
// 32-byte header and the two arrays, uploaded as they are and checked by the
// CSR check every upload runs.
#include <cstdio>
#include <cstring>
#include <vector>

#include "cds_gen.h"
#include "device_util.cuh"
#include "pipeline.h"

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t SMEM_SORT = 8192;  // row entries sorted in shared memory (32 KB)
constexpr uint32_t SORT_THREADS = 512;

__device__ __forceinline__ bool is_digit(uint8_t c) { return c >= '0' && c <= '9'; }
__device__ __forceinline__ bool is_space(uint8_t c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

// bad[0] |= 1 for a byte that is neither a digit nor a separator; start[i]
// = 1 when byte i starts a token; nl[i] = 1 for a newline byte
__global__ void k_scan_bytes(const uint8_t *__restrict__ txt, uint64_t len, uint32_t *__restrict__ start,
                             uint32_t *__restrict__ nl, uint32_t *__restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t c = txt[i];
    const bool d = is_digit(c);
    if (!d && !is_space(c)) atomicOr(bad, 1u);
    start[i] = d && (i == 0 || !is_digit(txt[i - 1]));
    nl[i] = c == '\n';
  }
}

// token t: its first byte pos[t] (compacted from the start flags with their
// exclusive scan), and its line: the number of newlines before it
__global__ void k_tokens(const uint32_t *__restrict__ start, const uint64_t *__restrict__ tok_at,
                         const uint64_t *__restrict__ line_at, uint64_t len, uint64_t *__restrict__ pos,
                         uint64_t *__restrict__ line) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (start[i]) {
      const uint64_t t = tok_at[i];
      pos[t] = i;
      line[t] = line_at[i];
    }
}

// value of each token (bad[0] |= 2 when it passes 2^32 - 1)
__global__ void k_values(const uint8_t *__restrict__ txt, uint64_t len, const uint64_t *__restrict__ pos,
                         uint64_t ntok, uint32_t *__restrict__ val, uint32_t *__restrict__ bad) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t x = 0;
    uint64_t i = pos[t];
    int digits = 0;
    while (i < len && is_digit(txt[i]) && digits <= 10) {
      x = x * 10 + (txt[i] - '0');
      i++;
      digits++;
    }
    if (x > 0xFFFFFFFFull) {
      atomicOr(bad, 2u);
      x = 0;
    }
    val[t] = (uint32_t)x;
  }
}

// Line starts: f[t] = 1 for the first token of a line; their compacted
// positions are sorted, so every token finds its line's first token (the
// vertex of a vertex line) by binary search.
__global__ void k_line_start_flags(const uint64_t *__restrict__ line, uint64_t ntok, uint32_t *__restrict__ f) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x)
    f[t] = t == 0 || line[t - 1] != line[t];
}
__global__ void k_line_start_fill(const uint32_t *__restrict__ f, const uint64_t *__restrict__ at, uint64_t ntok,
                                  uint64_t *__restrict__ starts) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x)
    if (f[t]) starts[at[t]] = t;
}

// head[t]: the first token of t's line (the last line start <= t)
__global__ void k_heads_of(const uint64_t *__restrict__ starts, uint64_t nstarts, uint64_t ntok,
                           uint64_t *__restrict__ head) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = nstarts;
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (starts[mid] <= t) lo = mid;
      else hi = mid;
    }
    head[t] = starts[lo];
  }
}

// degrees: each edge token (v, w), w != v, counts for v and for w
__global__ void k_edge_degrees(const uint32_t *__restrict__ val, const uint64_t *__restrict__ head,
                               uint64_t first_tok, uint64_t ntok, uint32_t n, uint32_t *__restrict__ deg,
                               uint32_t *__restrict__ bad) {
  for (uint64_t t = first_tok + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = head[t];
    const uint32_t v = val[h];
    if (v >= n) {
      atomicOr(bad, 4u);
      continue;
    }
    if (h == t) continue;
    const uint32_t w = val[t];
    if (w >= n) {
      atomicOr(bad, 4u);
      continue;
    }
    if (w == v) continue;
    atomicAdd(&deg[v], 1u);
    atomicAdd(&deg[w], 1u);
  }
}

__global__ void k_edge_scatter(const uint32_t *__restrict__ val, const uint64_t *__restrict__ head,
                               uint64_t first_tok, uint64_t ntok, uint32_t n, const uint64_t *__restrict__ roff,
                               uint32_t *__restrict__ cur, uint32_t *__restrict__ rows) {
  for (uint64_t t = first_tok + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntok;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = head[t];
    if (h == t) continue;
    const uint32_t v = val[h], w = val[t];
    if (v >= n || w >= n || w == v) continue;
    rows[roff[v] + atomicAdd(&cur[v], 1u)] = w;
    rows[roff[w] + atomicAdd(&cur[w], 1u)] = v;
  }
}

// Sort row r (one block) ascending, then count its distinct entries.
// Bitonic network over the row padded to a power of two with NONE; the
// padding of rows above SMEM_SORT lives in `spill` (one slab per block).
__device__ void bitonic(uint32_t *a, uint32_t m) {
  for (uint32_t size = 2; size <= m; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < m / 2; i += blockDim.x) {
        const uint32_t lo = 2 * i - (i & (stride - 1));
        const uint32_t hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint32_t x = a[lo], y = a[hi];
        if ((x > y) == up) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_rows(const uint64_t *__restrict__ roff, uint32_t n,
                                                             uint32_t *__restrict__ rows,
                                                             uint32_t *__restrict__ spill, uint64_t spill_slab,
                                                             uint32_t *__restrict__ ndeg) {
  __shared__ uint32_t s[SMEM_SORT];
  for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
    const uint64_t b = roff[r], e = roff[r + 1];
    const uint32_t len = (uint32_t)(e - b);
    if (len == 0) {
      if (threadIdx.x == 0) ndeg[r] = 0;
      continue;
    }
    uint32_t m = 1;
    while (m < len) m <<= 1;
    uint32_t *a = m <= SMEM_SORT ? s : spill + (uint64_t)blockIdx.x * spill_slab;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) a[i] = i < len ? rows[b + i] : NONE;
    __syncthreads();
    bitonic(a, m);
    // distinct values, written back in place (a stable compaction per block)
    uint32_t base = 0;
    for (uint32_t i0 = 0; i0 < len; i0 += blockDim.x) {
      const uint32_t i = i0 + threadIdx.x;
      const bool keep = i < len && (i == 0 || a[i] != a[i - 1]);
      uint32_t total;
      const uint32_t at = block_exclusive_scan<uint32_t>(keep ? 1u : 0u, &total);
      if (keep) rows[b + base + at] = a[i];
      base += total;
      __syncthreads();
    }
    if (threadIdx.x == 0) ndeg[r] = base;
    __syncthreads();
  }
}

__global__ void k_compact_rows(const uint64_t *__restrict__ roff, const uint64_t *__restrict__ off, uint32_t n,
                               const uint32_t *__restrict__ rows, uint32_t *__restrict__ adj) {
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = roff[v], o = off[v], d = off[v + 1] - o;
    for (uint64_t i = lane_id(); i < d; i += 32) adj[o + i] = rows[b + i];
  }
}

}  // namespace

namespace cds {

// Parses adjacency-list text (bytes already on the device) into a canonical
// CSR owned by a new graph.  Throws CDS_ERR_INPUT on malformed text.
void parse_adjlist_device(cds_ctx *c, cudaStream_t s, const uint8_t *txt, uint64_t len, cds_graph **out) {
  const int G = c->sm_count * 8;
  if (len >= 0xFFFFFFFFull * 4) fail(CDS_ERR_INPUT, "adjacency list too large");
  DBuf<uint32_t> start(c, s, len + 1), nl(c, s, len + 1), bad(c, s, 1);
  bad.zero();
  k_scan_bytes<<<G, 256, 0, s>>>(txt, len, start.p, nl.p, bad.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  DBuf<uint64_t> tok_at(c, s, len + 1), line_at(c, s, len + 1);
  scan_u32(start.p, tok_at.p, len, c, s);
  scan_u32(nl.p, line_at.p, len, c, s);
  uint64_t ntok = 0;
  uint32_t hbad = 0;
  {
    HostReads r(s);
    r.add(&ntok, tok_at.p + len);
    r.add(&hbad, bad.p);
    r.wait();
  }
  if (hbad) fail(CDS_ERR_INPUT, "adjacency list holds a byte that is not a digit or a separator");
  if (ntok < 2) fail(CDS_ERR_INPUT, "adjacency list lacks its header line");
  DBuf<uint64_t> pos(c, s, ntok), line(c, s, ntok);
  k_tokens<<<G, 256, 0, s>>>(start.p, tok_at.p, line_at.p, len, pos.p, line.p);
  start.release();
  nl.release();
  tok_at.release();
  line_at.release();
  DBuf<uint32_t> val(c, s, ntok);
  k_values<<<G, 256, 0, s>>>(txt, len, pos.p, ntok, val.p, bad.p);
  count_launch(2);
  CDS_CUDA(cudaGetLastError());
  // line starts (token indices), then every token's line head
  DBuf<uint32_t> lf(c, s, ntok);
  DBuf<uint64_t> lat(c, s, ntok + 1);
  k_line_start_flags<<<G, 256, 0, s>>>(line.p, ntok, lf.p);
  count_launch();
  scan_u32(lf.p, lat.p, ntok, c, s);
  uint64_t nlines = 0;
  uint32_t hdr[2] = {0, 0};
  uint64_t l0[2] = {0, 0};
  {
    HostReads r(s);
    r.add(&nlines, lat.p + ntok);
    r.add(hdr, val.p, 2);
    r.add(l0, line.p, 2);
    r.add(&hbad, bad.p);
    r.wait();
  }
  if (hbad) fail(CDS_ERR_INPUT, "adjacency list holds a number above 2^32 - 1");
  if (l0[0] != l0[1]) fail(CDS_ERR_INPUT, "the header line must hold n and m");
  const uint32_t n = hdr[0];
  DBuf<uint64_t> starts(c, s, nlines + 1), head(c, s, ntok);
  k_line_start_fill<<<G, 256, 0, s>>>(lf.p, lat.p, ntok, starts.p);
  k_heads_of<<<G, 256, 0, s>>>(starts.p, nlines, ntok, head.p);
  count_launch(2);
  lf.release();
  lat.release();
  // the header's tokens are not edges: the first edge token follows them
  uint64_t first_tok = 0;
  {
    std::vector<uint64_t> st(nlines > 1 ? 2 : 1);
    HostReads r(s);
    r.add(st.data(), starts.p, st.size());
    r.wait();
    first_tok = nlines > 1 ? st[1] : ntok;
  }
  DBuf<uint32_t> deg(c, s, (size_t)n + 1);
  deg.zero();
  k_edge_degrees<<<G, 256, 0, s>>>(val.p, head.p, first_tok, ntok, n, deg.p, bad.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  DBuf<uint64_t> roff(c, s, (size_t)n + 1);
  scan_u32(deg.p, roff.p, n, c, s);
  uint64_t slots = 0;
  uint32_t maxrow = 0;
  {
    HostReads r(s);
    r.add(&slots, roff.p + n);
    r.add(&hbad, bad.p);
    r.wait();
  }
  if (hbad & 4u) fail(CDS_ERR_INPUT, "adjacency list names a vertex id >= n");
  DBuf<uint32_t> rows(c, s, slots + 1), cur(c, s, (size_t)n + 1);
  cur.zero();
  k_edge_scatter<<<G, 256, 0, s>>>(val.p, head.p, first_tok, ntok, n, roff.p, cur.p, rows.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  val.release();
  head.release();
  pos.release();
  line.release();
  // the longest row sizes the spill slabs of rows sorted in global memory
  {
    std::vector<uint32_t> hd(n);
    if (n) {
      HostReads r(s);
      r.add(hd.data(), deg.p, n);
      r.wait();
    }
    for (uint32_t v = 0; v < n; v++) maxrow = std::max(maxrow, hd[v]);
  }
  uint64_t slab = 1;
  while (slab < maxrow) slab <<= 1;
  const uint32_t sort_grid = (uint32_t)c->sm_count * 2;
  DBuf<uint32_t> spill(c, s, slab > SMEM_SORT ? slab * sort_grid : 1);
  DBuf<uint32_t> ndeg(c, s, (size_t)n + 1);
  if (n) {
    k_sort_rows<<<sort_grid, SORT_THREADS, 0, s>>>(roff.p, n, rows.p, spill.p, slab, ndeg.p);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
  spill.release();
  cds_graph *g = new cds_graph();
  g->ctx = c;
  g->n = n;
  try {
    g->d_off = (uint64_t *)dalloc_bytes(c, ((size_t)n + 1) * 8, s);
    scan_u32(ndeg.p, g->d_off, n, c, s);
    uint64_t nnz = 0;
    {
      HostReads r(s);
      r.add(&nnz, g->d_off + n);
      r.wait();
    }
    g->nnz = nnz;
    g->d_adj = (uint32_t *)dalloc_bytes(c, (size_t)nnz * 4 + 16, s);
    if (n) {
      k_compact_rows<<<G, 256, 0, s>>>(roff.p, g->d_off, n, rows.p, g->d_adj);
      count_launch();
      CDS_CUDA(cudaGetLastError());
    }
    uint32_t maxd = 0;
    {
      std::vector<uint32_t> hd(n);
      if (n) {
        HostReads r(s);
        r.add(hd.data(), ndeg.p, n);
        r.wait();
      }
      for (uint32_t v = 0; v < n; v++) maxd = std::max(maxd, hd[v]);
    }
    g->max_degree = maxd;
    CDS_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    if (g->d_off) dfree(c, g->d_off, s);
    if (g->d_adj) dfree(c, g->d_adj, s);
    delete g;
    throw;
  }
  *out = g;
}

}  // namespace cds
