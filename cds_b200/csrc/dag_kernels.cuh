// dag_kernels.cuh -- device code of the DAG orientation (see dag.cu).
#pragma once
#include "device_util.cuh"

namespace {

__global__ void k_degree(const uint64_t *__restrict__ off, uint32_t n, uint32_t *__restrict__ deg) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
}

__device__ __forceinline__ bool above(uint32_t dw, uint32_t w, uint32_t dv, uint32_t v) {
  return dw > dv || (dw == dv && w > v);
}

// Warp per vertex, four groups of 32 neighbours in flight at a time: a hub's
// list is a chain of dependent loads (neighbour, then its degree), so this
// quarters the chain that bounds the kernel.
constexpr int DAG_U = 4;

__global__ void k_outdeg(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                         const uint32_t *__restrict__ deg, uint32_t n,
                         uint32_t *__restrict__ outdeg, uint32_t *__restrict__ maxout) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  uint32_t local_max = 0;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = off[v], e = off[v + 1];
    const uint32_t dv = (uint32_t)(e - b);
    uint32_t c = 0;
    for (uint64_t i0 = b + lane_id(); i0 < e; i0 += 32 * DAG_U) {
      uint32_t w[DAG_U];
#pragma unroll
      for (int u = 0; u < DAG_U; u++) w[u] = i0 + 32u * u < e ? adj[i0 + 32u * u] : 0xFFFFFFFFu;
#pragma unroll
      for (int u = 0; u < DAG_U; u++)
        if (w[u] != 0xFFFFFFFFu) c += above(deg[w[u]], w[u], dv, v);
    }
    c = warp_sum(c);
    if (lane_id() == 0) outdeg[v] = c;
    local_max = c > local_max ? c : local_max;
  }
  if (lane_id() == 0 && local_max) atomicMax(maxout, local_max);
}

// warp per vertex; writes the out-list in ascending id order plus padding
__global__ void k_dag_fill(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                           const uint32_t *__restrict__ deg, uint32_t n,
                           const uint64_t *__restrict__ doff, uint32_t *__restrict__ dadj) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = off[v], e = off[v + 1];
    const uint32_t dv = (uint32_t)(e - b);
    uint64_t w0 = doff[v];
    const uint64_t wend = doff[v + 1];
    for (uint64_t i0 = b; i0 < e; i0 += 32 * DAG_U) {
      uint32_t w[DAG_U];
      bool keep[DAG_U];
#pragma unroll
      for (int u = 0; u < DAG_U; u++) {
        const uint64_t i = i0 + 32u * u + lane_id();
        w[u] = i < e ? adj[i] : 0u;
      }
#pragma unroll
      for (int u = 0; u < DAG_U; u++) {
        const uint64_t i = i0 + 32u * u + lane_id();
        keep[u] = i < e && above(deg[w[u]], w[u], dv, v);
      }
      // groups in order, lanes in order within a group: ascending ids
#pragma unroll
      for (int u = 0; u < DAG_U; u++) {
        const uint32_t m = __ballot_sync(CDS_FULL, keep[u]);
        if (keep[u]) dadj[w0 + __popc(m & ((1u << lane_id()) - 1u))] = w[u];
        w0 += __popc(m);
      }
    }
    for (uint64_t i = w0 + lane_id(); i < wend; i += 32) dadj[i] = 0xFFFFFFFFu;
  }
}

}  // namespace
