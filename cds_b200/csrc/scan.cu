// scan.cu -- device-wide exclusive scan.  out has n+1 entries; out[n] =
// total.  Up to 65,536 values one block walks the input in order, carrying
// the running total (one launch: most scans here are over the vertices of
// one graph); larger inputs reduce tiles, scan the tile sums recursively
// and add the tile offsets.
#include "cds_internal.h"
#include "device_util.cuh"

namespace {

struct LoadU32 {
  const uint32_t *p;
  __device__ uint64_t operator()(size_t i) const { return p[i]; }
};
struct LoadU64 {
  const uint64_t *p;
  __device__ uint64_t operator()(size_t i) const { return p[i]; }
};
struct LoadPad4 {
  const uint32_t *p;
  __device__ uint64_t operator()(size_t i) const { return (p[i] + 3u) & ~3u; }
};

// Scans one tile per block into out (tile-local exclusive prefix) and writes
// the tile total to sums[blockIdx.x].
template <class L>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(L load, uint64_t *out,
                                                             uint64_t *sums, size_t n) {
  const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS];
  uint64_t t = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = base + i < n ? load(base + i) : 0;
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

// One block over the input in tiles of SMALL_TILE, in order, carrying the
// running total (n <= SMALL_TILES * SMALL_TILE): 32 consecutive values per
// thread, so a graph of up to 16,384 vertices is one pass.
constexpr int SMALL_ITEMS = 32;
constexpr size_t SMALL_TILE = (size_t)SCAN_THREADS * SMALL_ITEMS;
constexpr size_t SMALL_TILES = 4;
template <class L>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_small(L load, uint64_t *out, size_t n) {
  uint64_t carry = 0;
  for (size_t tile = 0; tile < n; tile += SMALL_TILE) {
    const size_t base = tile + (size_t)threadIdx.x * SMALL_ITEMS;
    uint64_t v[SMALL_ITEMS];
    uint64_t t = 0;
#pragma unroll
    for (int i = 0; i < SMALL_ITEMS; i++) {
      v[i] = base + i < n ? load(base + i) : 0;
      t += v[i];
    }
    uint64_t total;
    uint64_t ex = carry + block_exclusive_scan<uint64_t>(t, &total);
#pragma unroll
    for (int i = 0; i < SMALL_ITEMS; i++) {
      if (base + i < n) out[base + i] = ex;
      ex += v[i];
    }
    carry += total;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_scan_add(uint64_t *out, const uint64_t *tile_off, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tile_off[i / SCAN_TILE];
  if (i == 0) out[n] = tile_off[(n + SCAN_TILE - 1) / SCAN_TILE];
}

template <class L>
void scan_impl(L load, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s) {
  if (n == 0) {
    CDS_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
    return;
  }
  const size_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (n <= SMALL_TILES * SMALL_TILE) {
    k_scan_small<<<1, SCAN_THREADS, 0, s>>>(load, out, n);
    cds::count_launch();
    CDS_CUDA(cudaGetLastError());
    return;
  }
  cds::DBuf<uint64_t> sums(c, s, tiles);
  cds::DBuf<uint64_t> tile_off(c, s, tiles + 1);
  k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(load, out, sums.p, n);
  cds::count_launch();
  CDS_CUDA(cudaGetLastError());
  scan_impl(LoadU64{sums.p}, tile_off.p, tiles, c, s);
  k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, tile_off.p, n);
  cds::count_launch();
  CDS_CUDA(cudaGetLastError());
}

}  // namespace

namespace cds {
void scan_u32(const uint32_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s) {
  scan_impl(LoadU32{in}, out, n, c, s);
}
void scan_u64(const uint64_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s) {
  scan_impl(LoadU64{in}, out, n, c, s);
}
void scan_u32_pad4(const uint32_t *in, uint64_t *out, size_t n, cds_ctx *c, cudaStream_t s) {
  scan_impl(LoadPad4{in}, out, n, c, s);
}
}  // namespace cds
