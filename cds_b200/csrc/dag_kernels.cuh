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

// warp per vertex
__global__ void k_outdeg(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                         const uint32_t *__restrict__ deg, uint32_t n,
                         uint32_t *__restrict__ outdeg, uint32_t *__restrict__ maxout) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  uint32_t local_max = 0;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint64_t b = off[v], e = off[v + 1];
    const uint32_t dv = (uint32_t)(e - b);
    uint32_t c = 0;
    for (uint64_t i = b + lane_id(); i < e; i += 32) {
      const uint32_t w = adj[i];
      c += above(deg[w], w, dv, v);
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
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      const uint64_t i = i0 + lane_id();
      bool keep = false;
      uint32_t w = 0;
      if (i < e) {
        w = adj[i];
        keep = above(deg[w], w, dv, v);
      }
      const uint32_t m = __ballot_sync(CDS_FULL, keep);
      if (keep) dadj[w0 + __popc(m & ((1u << lane_id()) - 1u))] = w;
      w0 += __popc(m);
    }
    for (uint64_t i = w0 + lane_id(); i < wend; i += 32) dadj[i] = 0xFFFFFFFFu;
  }
}

}  // namespace
