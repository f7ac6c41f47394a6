// dag.cu -- orientation of the undirected CSR into a DAG.
//
// Replaces generateDAG (cudaCode/main.cu:22-57) with its kernels
// generateDegreeDAG / generateNeighborDAG (cudaCode/src/helpers.cu:112-173)
// and the host core ordering it depends on (cudaCode/src/graph.cpp:41-113).
// Each edge is oriented from the lower to the higher (degree, id) key, which
// bounds every out-degree by O(sqrt(m)) and needs no host-side ordering.  The
// k-clique set does not depend on the orientation.
//
// Out-lists keep ascending vertex ids and every row is padded to a multiple
// of 4 entries with 0xFFFFFFFF, so rows start on 16-byte boundaries and can
// be read with 128-bit loads.
#include "stages.h"
#include "device_util.cuh"

#include "dag_kernels.cuh"

namespace cds {

void build_dag(cds_ctx *c, cudaStream_t s, const uint64_t *off, const uint32_t *adj,
               uint32_t n, Dag &dag) {
  dag.n = n;
  dag.deg.alloc(n + 1);
  dag.outdeg.alloc(n + 1);
  dag.off.alloc(n + 1);
  DBuf<uint32_t> maxout(c, s, 1);
  maxout.zero();
  if (n) {
    const int grid = c->sm_count * 8;
    k_degree<<<grid, 256, 0, s>>>(off, n, dag.deg.p);
    k_outdeg<<<grid, 256, 0, s>>>(off, adj, dag.deg.p, n, dag.outdeg.p, maxout.p);
    count_launch(2);
    CDS_CUDA(cudaGetLastError());
  }
  scan_u32_pad4(dag.outdeg.p, dag.off.p, n, c, s);
  uint64_t total = 0;
  {
    HostReads r(s);
    r.add(&total, dag.off.p + n);
    r.add(&dag.max_out, maxout.p);
    r.wait();
  }
  dag.adj.alloc(total + 4);
  if (n) {
    k_dag_fill<<<c->sm_count * 8, 256, 0, s>>>(off, adj, dag.deg.p, n, dag.off.p, dag.adj.p);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
}

}  // namespace cds
