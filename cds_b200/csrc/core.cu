// core.cu -- densest core, edge pruning, connected components, and the
// component-local clique/incidence layout the flow stage reads.
//
// Replaces generateDensestCore (cudaCode/main.cu:345-399, helpers.cu:821-896),
// prune (main.cu:400-449, helpers.cu:898-1041), componentDecompose
// (main.cu:451-518, helpers.cu:937-978) and the clique bucketing of
// getConnectedComponentStatus / rearrangeCliqueData (helpers.cu:1043-1096),
// and on the CPU side locateDensestCore, cliqueEnumerationListRecord,
// pruneInvalidEdges and connectedComponentDecompose
// (cpuCode/c++/src/helpers.cpp:710-1116).
//
//  - The (k',Psi)-core is every vertex with core number >= k' where
//    k' = ceil(best core density); its cliques are the stored cliques whose
//    members are all in it, so nothing is listed a second time.
//  - Pruning marks each DAG arc covered by a core clique (clique records are
//    in orientation order, so member x -> member y is an arc for x < y).
//  - Components come from a lock-free union-find over the kept arcs (which
//    connect exactly what the core cliques connect) that always hangs the
//    larger root under the smaller one, so a component's root is its
//    smallest vertex and components are ordered as the reference's
//    ascending-start BFS orders them.
//  - Counters that many threads bump at once (per component, per instance)
//    are warp-aggregated: one atomic per distinct key in a warp.
#include "device_util.cuh"
#include "stages.h"
#include "pipeline.h"

#include <algorithm>

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t inst_of(const uint32_t *of_vertex, uint32_t v) {
  return of_vertex ? of_vertex[v] : 0u;
}

// Grid-stride loops below step whole warps (base is warp-uniform), because
// the warp-aggregated atomics need all 32 lanes.
__global__ void k_core_flags(const uint32_t *__restrict__ core, uint32_t n,
                             const uint32_t *__restrict__ of_vertex,
                             const unsigned long long *__restrict__ kp, uint8_t *__restrict__ in_core,
                             unsigned long long *__restrict__ core_size) {
  for (uint32_t b = blockIdx.x * blockDim.x; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t v = b + threadIdx.x;
    uint32_t i = 0;
    bool in = false;
    if (v < n) {
      i = inst_of(of_vertex, v);
      const unsigned long long t = kp[i];
      in = t > 0 && (unsigned long long)core[v] >= t;
      in_core[v] = in;
    }
    agg_add_u64(core_size, i, in);
  }
}

// A clique lies in the (k',Psi)-core when its smallest member core (cmin,
// from the peel) is at least its instance's k' > 0; the flag overwrites cmin.
// One instance: no record is read at all.
__global__ void k_clique_flags(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                               const unsigned long long *__restrict__ kp, uint32_t *__restrict__ flag,
                               const uint32_t *__restrict__ of_vertex,
                               unsigned long long *__restrict__ core_cliques) {
  const unsigned long long kp0 = kp[0];
  RunCount run;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < m; b += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = b + threadIdx.x;
    bool in = false;
    uint32_t i = 0;
    if (c < m) {
      i = inst_of(of_vertex, of_vertex ? members[c * k] : 0u);
      const unsigned long long t = of_vertex ? kp[i] : kp0;
      in = t > 0 && (unsigned long long)flag[c] >= t;
      flag[c] = in;
    }
    run.add(core_cliques, i, in);
  }
  run.flush(core_cliques);
}

// arc u -> w of the DAG (w in the out-list of u), or NONE
__device__ __forceinline__ uint64_t find_arc(const uint64_t *doff, const uint32_t *dadj,
                                             const uint32_t *outdeg, uint32_t u, uint32_t w) {
  uint64_t lo = doff[u], hi = lo + outdeg[u];
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (dadj[mid] < w) lo = mid + 1;
    else hi = mid;
  }
  return (lo < doff[u] + outdeg[u] && dadj[lo] == w) ? lo : ~0ull;
}

__global__ void k_mark_arcs(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                            const uint32_t *__restrict__ flag, const uint64_t *__restrict__ doff,
                            const uint32_t *__restrict__ dadj, const uint32_t *__restrict__ outdeg,
                            uint8_t *__restrict__ arc_keep, uint32_t *__restrict__ err) {
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m;
       c += (uint64_t)gridDim.x * blockDim.x) {
    if (!flag[c]) continue;
    const uint32_t *r = members + c * k;
    for (uint32_t x = 0; x < k; x++)
      for (uint32_t y = x + 1; y < k; y++) {
        const uint64_t a = find_arc(doff, dadj, outdeg, r[x], r[y]);
        if (a == ~0ull) atomicOr(err, DEV_ERR_INTERNAL);
        else arc_keep[a] = 1;
      }
  }
}

// Small cores (at most PAIR_CORE_MAX vertices in all): the pairs that core
// cliques cover are marked in a bitmap over core-local ids -- a read, and an
// atomic only for a bit not yet set -- instead of a binary search for each
// of a clique's k(k-1)/2 arcs; a dense core's cliques share their pairs
// thousands of times over.  Then every DAG arc between core vertices looks
// its pair up.
constexpr uint32_t PAIR_CORE_MAX = 4096;

// core-local ids in vertex order: f[v] = in_core[v], scanned into lid, and
// the inverse core_vertex[lid] = v (so the smallest id of a set of core
// vertices is its smallest vertex)
__global__ void k_core_u32(const uint8_t *__restrict__ in_core, uint32_t n, uint32_t *__restrict__ f) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) f[v] = in_core[v];
}
__global__ void k_core_vertex(const uint8_t *__restrict__ in_core, const uint64_t *__restrict__ lid, uint32_t n,
                              uint32_t *__restrict__ core_vertex) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (in_core[v]) core_vertex[lid[v]] = v;
}

// Components of a small core in one block: union-find over the covered
// pairs of the bitmap with the parents in shared memory (smaller id wins, so
// a root is its component's smallest vertex); root[i] = the root of core id i.
__device__ __forceinline__ uint32_t s_find(uint32_t *par, uint32_t x) {
  uint32_t p = par[x];
  while (p != x) {
    const uint32_t gp = par[p];
    if (gp != p) par[x] = gp;
    x = p;
    p = gp;
  }
  return x;
}
__global__ void __launch_bounds__(1024) k_small_components(const uint32_t *__restrict__ bits, uint32_t words,
                                                           uint32_t ncore, uint32_t *__restrict__ root,
                                                           uint32_t *__restrict__ err) {
  __shared__ uint32_t par[PAIR_CORE_MAX];
  for (uint32_t i = threadIdx.x; i < ncore; i += blockDim.x) par[i] = i;
  __syncthreads();
  const uint64_t total = (uint64_t)ncore * words;
  for (uint64_t w = threadIdx.x; w < total; w += blockDim.x) {
    uint32_t word = bits[w];
    const uint32_t a0 = (uint32_t)(w / words), b0 = (uint32_t)(w % words) * 32;
    while (word) {
      const uint32_t b = b0 + (uint32_t)(__ffs(word) - 1);
      word &= word - 1;
      uint32_t a = a0, bb = b;
      for (int tries = 0;; tries++) {
        if (tries > (1 << 20)) {
          atomicOr(err, DEV_ERR_TIMEOUT);
          break;
        }
        const uint32_t ra = s_find(par, a), rb = s_find(par, bb);
        if (ra == rb) break;
        const uint32_t lo = ra < rb ? ra : rb, hi = ra < rb ? rb : ra;
        if (atomicCAS(&par[hi], hi, lo) == hi) break;
        a = lo;
        bb = hi;
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < ncore; i += blockDim.x) {
    uint32_t r = i;
    while (par[r] != r) r = par[r];
    root[i] = r;
  }
}

__global__ void k_comp_from_roots(const uint8_t *__restrict__ in_core, const uint64_t *__restrict__ lid,
                                  const uint32_t *__restrict__ root, const uint32_t *__restrict__ core_vertex,
                                  uint32_t n, uint32_t *__restrict__ comp) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    comp[v] = in_core[v] ? core_vertex[root[lid[v]]] : NONE;
}

__global__ void k_mark_pairs(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                             const uint32_t *__restrict__ flag, const uint64_t *__restrict__ lid,
                             uint32_t words, uint32_t *__restrict__ bits) {
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m;
       c += (uint64_t)gridDim.x * blockDim.x) {
    if (!flag[c]) continue;
    auto mark = [&](uint32_t a, uint32_t b) {
      uint32_t *w = bits + (uint64_t)a * words + (b >> 5);
      const uint32_t bit = 1u << (b & 31);
      if (!(*(volatile uint32_t *)w & bit)) atomicOr(w, bit);
    };
    if (k == 4) {  // the record in one 16-byte load, its local ids gathered together
      const uint4 q = *reinterpret_cast<const uint4 *>(members + c * 4);
      const uint32_t a0 = (uint32_t)lid[q.x], a1 = (uint32_t)lid[q.y], a2 = (uint32_t)lid[q.z],
                     a3 = (uint32_t)lid[q.w];
      mark(a0, a1);
      mark(a0, a2);
      mark(a0, a3);
      mark(a1, a2);
      mark(a1, a3);
      mark(a2, a3);
      continue;
    }
    const uint32_t *r = members + c * k;
    for (uint32_t x = 0; x < k; x++) {
      const uint32_t a = (uint32_t)lid[r[x]];
      for (uint32_t y = x + 1; y < k; y++) mark(a, (uint32_t)lid[r[y]]);
    }
  }
}

__global__ void k_pairs_to_arcs(const uint64_t *__restrict__ doff, const uint32_t *__restrict__ dadj,
                                const uint32_t *__restrict__ outdeg, const uint8_t *__restrict__ in_core,
                                const uint64_t *__restrict__ lid, uint32_t n, uint32_t words,
                                const uint32_t *__restrict__ bits, uint8_t *__restrict__ arc_keep) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    if (!in_core[u]) continue;
    const uint32_t a = (uint32_t)lid[u];
    for (uint32_t t = lane_id(); t < outdeg[u]; t += 32) {
      const uint32_t w = dadj[doff[u] + t];
      if (!in_core[w]) continue;
      const uint32_t b = (uint32_t)lid[w];
      if (bits[(uint64_t)a * words + (b >> 5)] & (1u << (b & 31))) arc_keep[doff[u] + t] = 1;
    }
  }
}

// warp per vertex: kept arcs per instance
__global__ void k_count_arcs(const uint64_t *__restrict__ doff, const uint32_t *__restrict__ outdeg,
                             const uint8_t *__restrict__ arc_keep, uint32_t n,
                             const uint32_t *__restrict__ of_vertex,
                             unsigned long long *__restrict__ out) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    uint32_t c = 0;
    for (uint32_t t = lane_id(); t < outdeg[v]; t += 32) c += arc_keep[doff[v] + t];
    c = warp_sum(c);
    if (lane_id() == 0 && c) atomicAdd(&out[inst_of(of_vertex, v)], (unsigned long long)c);
  }
}

__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x) {
  uint32_t p = parent[x];
  while (p != x) {
    const uint32_t gp = parent[p];
    if (gp != p) parent[x] = gp;  // path halving; only ever points closer to the root
    x = p;
    p = gp;
  }
  return x;
}

// union-find over the kept arcs: they connect exactly what the core cliques
// connect, with at most m unions instead of (k-1)|Psi|
__global__ void k_union(const uint64_t *__restrict__ doff, const uint32_t *__restrict__ dadj,
                        const uint32_t *__restrict__ outdeg, const uint8_t *__restrict__ keep,
                        uint32_t n, uint32_t *parent, uint32_t *err) {
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    for (uint32_t t = lane_id(); t < outdeg[u]; t += 32) {
      if (!keep[doff[u] + t]) continue;
      uint32_t a = u, b = dadj[doff[u] + t];
      for (int tries = 0;; tries++) {
        if (tries > (1 << 20)) {
          atomicOr(err, DEV_ERR_TIMEOUT);
          break;
        }
        const uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
        if (ra == rb) break;
        const uint32_t lo = ra < rb ? ra : rb, hi = ra < rb ? rb : ra;
        if (atomicCAS(&parent[hi], hi, lo) == hi) break;
        a = lo;
        b = hi;
      }
    }
  }
}

__global__ void k_roots(uint32_t *parent, const uint8_t *__restrict__ in_core, uint32_t n,
                        uint32_t *__restrict__ comp) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    comp[v] = in_core[v] ? uf_find(parent, v) : NONE;
}

// Core cliques per component: the records are stored by root vertex
// (cliques [base[u], base[u+1]) have u first), and a core clique lies in its
// root's component, so only the flags are read -- no record.  A warp takes
// a chunk of clique indices (a hub root's range of tens of millions of
// cliques is shared by many warps; `chunk` shrinks with the clique count so
// that small problems still have a chunk per warp and few roots per chunk),
// finds the chunk's first root by binary search, and adds the flag sum of
// each root's part of the chunk to that root's component.
__global__ void k_comp_cliques(const unsigned long long *__restrict__ base, uint32_t n, uint64_t m,
                               uint32_t chunk, const uint32_t *__restrict__ flag,
                               const uint32_t *__restrict__ comp, unsigned long long *__restrict__ ccount) {
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint64_t nchunks = (m + chunk - 1) / chunk;
  for (uint64_t ch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ch < nchunks; ch += warps) {
    uint64_t c0 = ch * chunk;
    const uint64_t c1 = min(m, c0 + chunk);
    // the last root u with base[u] <= c0 (base[0] = 0, base[n] = m)
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (base[mid] <= c0) lo = mid;
      else hi = mid;
    }
    uint32_t u = lo;
    while (c0 < c1) {
      const uint64_t e = min(c1, (uint64_t)base[u + 1]);
      const uint32_t r = comp[u];
      if (e > c0 && r != NONE) {  // a root outside the core has no core clique
        unsigned long long cnt = 0;
        for (uint64_t c = c0 + lane_id(); c < e; c += 32) cnt += flag[c];
        cnt = warp_sum(cnt);
        if (lane_id() == 0 && cnt) atomicAdd(&ccount[r], cnt);
      }
      c0 = e;
      u++;
    }
  }
}

// roots of components with >= 1 clique; component counts per instance
__global__ void k_root_flags(const uint32_t *__restrict__ comp, const unsigned long long *__restrict__ ccount,
                             uint32_t n, const uint32_t *__restrict__ of_vertex,
                             uint32_t *__restrict__ is_root, unsigned long long *__restrict__ ncomp) {
  for (uint32_t b = blockIdx.x * blockDim.x; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t v = b + threadIdx.x;
    bool root = false;
    if (v < n) {
      root = comp[v] == v;
      is_root[v] = root && ccount[v] > 0;
    }
    agg_add_u64(ncomp, root ? inst_of(of_vertex, v) : 0u, root);
  }
}

__global__ void k_comp_sizes(const uint32_t *__restrict__ comp, const uint64_t *__restrict__ cidx,
                             const unsigned long long *__restrict__ ccount, uint32_t n,
                             uint32_t *__restrict__ csize, unsigned long long *__restrict__ cclq,
                             const uint32_t *__restrict__ core, uint32_t *__restrict__ cmax) {
  for (uint32_t b = blockIdx.x * blockDim.x; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t v = b + threadIdx.x;
    bool in = false;
    uint32_t ci = 0;
    if (v < n) {
      const uint32_t r = comp[v];
      in = r != NONE && ccount[r] > 0;
      if (in) {
        ci = (uint32_t)cidx[r];
        if (r == v) cclq[ci] = ccount[r];
      }
    }
    agg_inc(csize, ci, in);
    const uint32_t grp = __match_any_sync(CDS_FULL, in ? ci : NONE);
    const uint32_t mx = __reduce_max_sync(grp, in ? core[v] : 0u);
    if (in && (int)lane_id() == __ffs(grp) - 1) atomicMax(&cmax[ci], mx);
  }
}

__global__ void k_local_ids(const uint32_t *__restrict__ comp, const uint64_t *__restrict__ cidx,
                            const unsigned long long *__restrict__ ccount, uint32_t n,
                            const uint64_t *__restrict__ vbeg, uint32_t *__restrict__ vcur,
                            uint32_t *__restrict__ local, uint32_t *__restrict__ vmap,
                            uint32_t *__restrict__ vcnet) {
  for (uint32_t b = blockIdx.x * blockDim.x; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t v = b + threadIdx.x;
    bool in = false;
    uint32_t ci = 0;
    if (v < n) {
      const uint32_t r = comp[v];
      in = r != NONE && ccount[r] > 0;
      if (in) ci = (uint32_t)cidx[r];
      else local[v] = NONE;
    }
    const uint32_t slot = agg_inc(vcur, ci, in);
    if (in) {
      const uint32_t l = (uint32_t)vbeg[ci] + slot;
      local[v] = l;
      vmap[l] = v;
      vcnet[l] = ci;
    }
  }
}

// Networks of at most this many vertices (all components of a problem
// together) count per-vertex degrees and cursors per block in shared memory.
constexpr uint32_t SMALL_NV = 2048;

// Core cliques grouped by component, in the local ids of their networks.
// A block whose core cliques all lie in one component (the usual case) takes
// its slots with one atomic; otherwise each warp takes its own.
__global__ void k_bucket_cliques(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                                 const uint32_t *__restrict__ flag, const uint32_t *__restrict__ comp,
                                 const uint64_t *__restrict__ cidx, const uint64_t *__restrict__ cbeg,
                                 unsigned long long *__restrict__ ccur, const uint32_t *__restrict__ local,
                                 uint32_t nv, uint32_t *__restrict__ rec, uint32_t *__restrict__ ldeg) {
  __shared__ uint32_t s_lo, s_hi;
  __shared__ unsigned long long s_base;
  __shared__ uint32_t s_ldeg[SMALL_NV];  // this block's degree counts (nv <= SMALL_NV)
  const bool small = nv <= SMALL_NV;
  if (small) {
    for (uint32_t l = threadIdx.x; l < nv; l += blockDim.x) s_ldeg[l] = 0;
    __syncthreads();
  }
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < m; b += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = b + threadIdx.x;
    const bool in = c < m && flag[c];
    const uint32_t *r = members + (in ? c : 0) * k;
    const uint32_t ci = in ? (uint32_t)cidx[comp[r[0]]] : 0u;
    if (threadIdx.x == 0) {
      s_lo = 0xFFFFFFFFu;
      s_hi = 0;
    }
    __syncthreads();
    const uint32_t lo = warp_min(in ? ci : 0xFFFFFFFFu), hi = warp_max(in ? ci : 0u);
    if (lane_id() == 0) {
      atomicMin(&s_lo, lo);
      atomicMax(&s_hi, hi);
    }
    __syncthreads();
    unsigned long long slot;
    if (s_lo == s_hi) {  // one component in the block (s_lo > s_hi: none)
      uint32_t total;
      const uint32_t rank = block_exclusive_scan<uint32_t>(in ? 1u : 0u, &total);
      if (threadIdx.x == 0) s_base = atomicAdd(&ccur[s_lo], (unsigned long long)total);
      __syncthreads();
      slot = s_base + rank;
    } else {
      slot = agg_inc_u64(ccur, ci, in);
    }
    const uint64_t pos = in ? cbeg[ci] + slot : 0;
    // the rest of the record (spare slots, flow words) starts at zero, so
    // the first flow over these records needs no reset pass
    if (k <= 4) {
      // the whole record in 16-byte stores (one for k = 2, two for k = 3, 4)
      uint32_t l[4] = {0u, 0u, 0u, 0u};
      if (k == 4 && in) {
        const uint4 q = *reinterpret_cast<const uint4 *>(members + c * 4);
        l[0] = local[q.x];
        l[1] = local[q.y];
        l[2] = local[q.z];
        l[3] = local[q.w];
      } else if (in) {
        for (uint32_t j = 0; j < k; j++) l[j] = local[r[j]];
      }
#pragma unroll
      for (uint32_t j = 0; j < 4; j++)
        if (j < k) agg_add_u32(small ? s_ldeg : ldeg, l[j], in);
      if (in) {
        uint4 *R = reinterpret_cast<uint4 *>(rec + (pos << rec_shift(k)));
        R[0] = make_uint4(l[0], l[1], l[2], l[3]);
        if (k > 2) R[1] = make_uint4(0u, 0u, 0u, 0u);
      }
    } else {
      for (uint32_t j = 0; j < k; j++) {
        const uint32_t l = in ? local[r[j]] : 0u;
        if (in) rec[(pos << rec_shift(k)) + j] = l;
        agg_add_u32(small ? s_ldeg : ldeg, l, in);
      }
      if (in)
        for (uint32_t j = k; j < 2 * rec_slots(k); j++) rec[(pos << rec_shift(k)) + j] = 0u;
    }
    __syncthreads();  // s_lo, s_hi and s_base are reused by the next tile
  }
  if (small)
    for (uint32_t l = threadIdx.x; l < nv; l += blockDim.x)
      if (s_ldeg[l]) atomicAdd(&ldeg[l], s_ldeg[l]);
}

template <typename I>
__global__ void k_fill_vinc(const uint32_t *__restrict__ rec, uint64_t nc, uint32_t k,
                            const uint64_t *__restrict__ vinc_off, uint32_t *__restrict__ cur,
                            I *__restrict__ vinc) {
  // slot-major walk (slot j of every clique, then slot j+1): lanes see the
  // same slot of consecutive cliques, which often share that member, so the
  // cursor atomics aggregate
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint32_t j = 0; j < k; j++) {
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < nc; b += stride) {
      const uint64_t c = b + threadIdx.x;
      const bool in = c < nc;
      const uint32_t l = in ? rec[(c << rec_shift(k)) + j] : 0u;
      const uint32_t slot = agg_inc(cur, l, in);
      if (in) vinc[vinc_off[l] + slot] = (I)c;
    }
  }
}

// The same for networks of at most SMALL_NV vertices, where the per-vertex
// cursors would be a few hundred hot words: each block takes a contiguous
// range of cliques, counts its incidences per vertex in shared memory,
// reserves one range per vertex with a single atomic, then writes.
template <typename I>
__global__ void k_fill_vinc_small(const uint32_t *__restrict__ rec, uint64_t nc, uint32_t k, uint32_t nv,
                                  const uint64_t *__restrict__ vinc_off, uint32_t *__restrict__ cur,
                                  I *__restrict__ vinc) {
  __shared__ uint32_t s_cnt[SMALL_NV], s_base[SMALL_NV];
  const uint64_t per = (nc + gridDim.x - 1) / gridDim.x;
  const uint64_t c_lo = min(nc, (uint64_t)blockIdx.x * per), c_hi = min(nc, c_lo + per);
  for (uint32_t l = threadIdx.x; l < nv; l += blockDim.x) s_cnt[l] = 0;
  __syncthreads();
  // a thread per clique record (consecutive threads, consecutive records,
  // which share their first members: lanes in runs of one member reserve
  // together, not 32 conflicting atomics on one word)
  const uint32_t rs = rec_shift(k);
  for (uint64_t c0 = c_lo; c0 < c_hi; c0 += blockDim.x) {
    const uint64_t c = c0 + threadIdx.x;
    const bool in = c < c_hi;
    for (uint32_t j = 0; j < k; j++) run_inc(s_cnt, in ? rec[(c << rs) + j] : 0u, in);
  }
  __syncthreads();
  for (uint32_t l = threadIdx.x; l < nv; l += blockDim.x) {
    const uint32_t n_l = s_cnt[l];
    s_base[l] = n_l ? atomicAdd(&cur[l], n_l) : 0u;
    s_cnt[l] = 0;
  }
  __syncthreads();
  for (uint64_t c0 = c_lo; c0 < c_hi; c0 += blockDim.x) {
    const uint64_t c = c0 + threadIdx.x;
    const bool in = c < c_hi;
    for (uint32_t j = 0; j < k; j++) {
      const uint32_t l = in ? rec[(c << rs) + j] : 0u;
      const uint32_t at = run_inc(s_cnt, l, in);
      if (in) vinc[vinc_off[l] + s_base[l] + at] = (I)c;
    }
  }
}

__global__ void k_iota(uint32_t *__restrict__ a, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) a[v] = v;
}

__global__ void k_gather_roots(const uint32_t *__restrict__ is_root, const uint64_t *__restrict__ cidx,
                               uint32_t n, uint32_t *__restrict__ roots) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (is_root[v]) roots[cidx[v]] = v;
}

}  // namespace

namespace cds {

void densest_core_and_components(cds_ctx *c, cudaStream_t s, const Dag &dag, const Cliques &cl,
                                 const PeelOut &pe, const Instances &inst, uint32_t k,
                                 CoreOut &out, bool need_networks, StageClock *clk) {
  const uint32_t n = dag.n;
  const uint64_t m = cl.count;
  const uint32_t ninst = inst.count;
  const uint32_t *of_vertex = ninst > 1 ? inst.of_vertex.p : nullptr;
  const int G = c->sm_count * 8;

  out.threshold.assign(ninst, 0);
  for (uint32_t i = 0; i < ninst; i++)
    if (pe.best_den[i] && pe.best_num[i])
      out.threshold[i] = (pe.best_num[i] + pe.best_den[i] - 1) / pe.best_den[i];
  DBuf<unsigned long long> kp(c, s, ninst);
  CDS_CUDA(cudaMemcpyAsync(kp.p, out.threshold.data(), ninst * 8, cudaMemcpyHostToDevice, s));
  DBuf<unsigned long long> stats(c, s, 4 * (size_t)ninst);  // core size, core cliques, arcs, comps
  stats.zero();
  DBuf<uint8_t> in_core(c, s, n + 1);
  uint32_t *flag = pe.cmin.p;  // becomes the core-clique flags
  DBuf<uint32_t> err(c, s, 1);
  err.zero();
  {
    ProfScope ps(c, s, "core_flags");
    if (n) k_core_flags<<<G, 256, 0, s>>>(pe.core.p, n, of_vertex, kp.p, in_core.p, stats.p);
    if (m) k_clique_flags<<<G, 256, 0, s>>>(cl.members.p, m, k, kp.p, flag, of_vertex, stats.p + ninst);
  }
  count_launch(2);
  CDS_CUDA(cudaGetLastError());
  if (clk) out.mk_core = clk->mark();

  // prune: arcs inside >= 1 core clique
  uint64_t ncore = 0;
  {
    std::vector<unsigned long long> h(ninst);
    HostReads r(s);
    r.add(h.data(), stats.p, ninst);
    r.wait();
    for (auto x : h) ncore += x;
  }
  DBuf<uint8_t> keep(c, s, dag.adj.n + 1);
  const bool small_core = m && n && ncore <= PAIR_CORE_MAX;
  const uint32_t words = (uint32_t)((ncore + 31) / 32);
  DBuf<uint64_t> lid(c, s, small_core ? n + 1 : 0);
  DBuf<uint32_t> core_vertex(c, s, small_core ? ncore + 1 : 0), bits(c, s, small_core ? ncore * words + 1 : 0);
  {
    keep.zero();
    ProfScope ps(c, s, "prune_arcs");
    if (small_core) {
      {
        DBuf<uint32_t> f(c, s, n + 1);
        k_core_u32<<<G, 256, 0, s>>>(in_core.p, n, f.p);
        scan_u32(f.p, lid.p, n, c, s);
      }
      bits.zero();
      k_core_vertex<<<G, 256, 0, s>>>(in_core.p, lid.p, n, core_vertex.p);
      k_mark_pairs<<<G, 256, 0, s>>>(cl.members.p, m, k, flag, lid.p, words, bits.p);
      k_pairs_to_arcs<<<G, 256, 0, s>>>(dag.off.p, dag.adj.p, dag.outdeg.p, in_core.p, lid.p, n, words, bits.p,
                                        keep.p);
      count_launch(4);
    } else if (m) {
      k_mark_arcs<<<G, 256, 0, s>>>(cl.members.p, m, k, flag, dag.off.p, dag.adj.p, dag.outdeg.p, keep.p,
                                    err.p);
      count_launch();
    }
    if (n) k_count_arcs<<<G, 256, 0, s>>>(dag.off.p, dag.outdeg.p, keep.p, n, of_vertex, stats.p + 2 * ninst);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
  if (clk) out.mk_prune = clk->mark();

  // components
  DBuf<uint32_t> parent(c, s, n + 1), comp(c, s, n + 1);
  DBuf<unsigned long long> ccount(c, s, n + 1);  // core cliques per component root (may pass 2^32)
  if (n) {
    k_iota<<<G, 256, 0, s>>>(parent.p, n);
    count_launch();
  }
  ccount.zero();
  DBuf<uint32_t> is_root(c, s, n + 1);
  DBuf<uint64_t> cidx(c, s, n + 1);
  {
    ProfScope ps_cc(c, s, "components_unionfind");
    if (small_core) {
      DBuf<uint32_t> root(c, s, ncore + 1);
      k_small_components<<<1, 1024, 0, s>>>(bits.p, words, (uint32_t)ncore, root.p, err.p);
      k_comp_from_roots<<<G, 256, 0, s>>>(in_core.p, lid.p, root.p, core_vertex.p, n, comp.p);
    } else if (n) {
      k_union<<<G, 256, 0, s>>>(dag.off.p, dag.adj.p, dag.outdeg.p, keep.p, n, parent.p, err.p);
      k_roots<<<G, 256, 0, s>>>(parent.p, in_core.p, n, comp.p);
    }
    if (m)
      k_comp_cliques<<<G, 256, 0, s>>>(reinterpret_cast<const unsigned long long *>(cl.base.p), n, m,
                                       (uint32_t)std::min<uint64_t>(8192, std::max<uint64_t>(64, m / (4ull * G * 8))),
                                       flag, comp.p, ccount.p);
    if (n) k_root_flags<<<G, 256, 0, s>>>(comp.p, ccount.p, n, of_vertex, is_root.p, stats.p + 3 * ninst);
  }
  count_launch(4);
  CDS_CUDA(cudaGetLastError());
  scan_u32(is_root.p, cidx.p, n, c, s);
  // one wait for the component count, the per-instance statistics and the status
  uint64_t ncomp64 = 0;
  uint32_t e0 = 0;
  {
    std::vector<unsigned long long> h(4 * (size_t)ninst);
    HostReads r(s);
    r.add(&ncomp64, cidx.p + n);
    r.add(&e0, err.p);
    r.add(h.data(), stats.p, h.size());
    r.wait();
    out.core_size.assign(h.begin(), h.begin() + ninst);
    out.core_cliques.assign(h.begin() + ninst, h.begin() + 2 * ninst);
    out.pruned_edges.assign(h.begin() + 2 * ninst, h.begin() + 3 * ninst);
    out.n_components.resize(ninst);
    for (uint32_t i = 0; i < ninst; i++) out.n_components[i] = (uint32_t)h[3 * ninst + i];
  }
  const uint32_t ncomp = (uint32_t)ncomp64;
  out.ncomp = ncomp;
  if (e0 & DEV_ERR_TIMEOUT) fail(CDS_ERR_TIMEOUT, "components: union-find retry budget exhausted");
  if (e0) fail(CDS_ERR_CUDA, "densest core: clique record is not a DAG path");

  out.comp_inst.assign(ncomp, 0);
  out.comp_vbeg.assign(ncomp + 1, 0);
  out.comp_cbeg.assign(ncomp + 1, 0);
  out.comp_maxcore.assign(ncomp, 0);
  out.comp_root.assign(ncomp, 0);
  if (!need_networks || ncomp == 0) return;
  DBuf<uint32_t> csize(c, s, ncomp), cmax(c, s, ncomp), roots(c, s, ncomp);
  DBuf<unsigned long long> cclq(c, s, ncomp);
  csize.zero();
  cclq.zero();
  cmax.zero();
  k_comp_sizes<<<G, 256, 0, s>>>(comp.p, cidx.p, ccount.p, n, csize.p, cclq.p, pe.core.p, cmax.p);
  k_gather_roots<<<G, 256, 0, s>>>(is_root.p, cidx.p, n, roots.p);
  count_launch(2);
  CDS_CUDA(cudaGetLastError());
  DBuf<uint64_t> vbeg(c, s, ncomp + 1), cbeg(c, s, ncomp + 1);
  scan_u32(csize.p, vbeg.p, ncomp, c, s);
  scan_u64(reinterpret_cast<const uint64_t *>(cclq.p), cbeg.p, ncomp, c, s);
  std::vector<uint64_t> hv(ncomp + 1), hc(ncomp + 1);
  std::vector<uint32_t> hroots(ncomp);
  {
    HostReads r(s);
    r.add(hv.data(), vbeg.p, ncomp + 1);
    r.add(hc.data(), cbeg.p, ncomp + 1);
    r.add(out.comp_maxcore.data(), cmax.p, ncomp);
    r.add(hroots.data(), roots.p, ncomp);
    r.wait();
  }
  for (uint32_t i = 0; i <= ncomp; i++) {
    out.comp_vbeg[i] = (uint32_t)hv[i];
    out.comp_cbeg[i] = hc[i];
  }
  out.comp_root = hroots;
  for (uint32_t i = 0; i < ncomp; i++) {
    uint32_t r = hroots[i], ii = 0;
    // instance of the root: binary search in the instance table
    ii = (uint32_t)(std::upper_bound(inst.h_vbeg.begin(), inst.h_vbeg.end(), r) - inst.h_vbeg.begin()) - 1;
    out.comp_inst[i] = ii;
  }
  const uint32_t nv = (uint32_t)hv[ncomp];
  const uint64_t nc = hc[ncomp];
  out.vmap.c = out.rec.c = out.vcnet.c = out.vinc_off.c = out.vinc.c = c;
  out.vmap.s = out.rec.s = out.vcnet.s = out.vinc_off.s = out.vinc.s = s;
  out.vmap.alloc(nv + 1);
  out.vcnet.alloc(nv + 1);
  out.rec.alloc((nc << rec_shift(k)) + 1);
  DBuf<uint32_t> local(c, s, n + 1), vcur(c, s, ncomp), ldeg(c, s, nv + 1);
  DBuf<unsigned long long> ccur(c, s, ncomp);
  vcur.zero();
  ccur.zero();
  ldeg.zero();
  {
    ProfScope ps_b(c, s, "components_bucket");
    k_local_ids<<<G, 256, 0, s>>>(comp.p, cidx.p, ccount.p, n, vbeg.p, vcur.p, local.p, out.vmap.p,
                                 out.vcnet.p);
    if (m) k_bucket_cliques<<<G, 256, 0, s>>>(cl.members.p, m, k, flag, comp.p, cidx.p, cbeg.p,
                                             ccur.p, local.p, nv, out.rec.p, ldeg.p);
  }
  count_launch(2);
  CDS_CUDA(cudaGetLastError());
  out.vinc_off.alloc(nv + 1);
  scan_u32(ldeg.p, out.vinc_off.p, nv, c, s);
  out.flows_zero = true;
  // each vertex's cliques as u32 record indices while they fit, else u64
  // (two words each); the vertex's slot in a record is found by matching
  out.vinc_wide = nc >= 0xFFFFFFFFull || (c->flags & CDS_CONFIG_WIDE_FLOW);
  out.vinc.alloc(nc * k * (out.vinc_wide ? 2 : 1) + 2);
  {
    ProfScope ps_v(c, s, "components_vinc");
    DBuf<uint32_t> cur(c, s, nv + 1);
    cur.zero();
    if (nc && nv <= SMALL_NV && out.vinc_wide)
      k_fill_vinc_small<uint64_t><<<G, 256, 0, s>>>(out.rec.p, nc, k, nv, out.vinc_off.p, cur.p,
                                                    reinterpret_cast<uint64_t *>(out.vinc.p));
    else if (nc && nv <= SMALL_NV)
      k_fill_vinc_small<uint32_t><<<G, 256, 0, s>>>(out.rec.p, nc, k, nv, out.vinc_off.p, cur.p, out.vinc.p);
    else if (nc && out.vinc_wide)
      k_fill_vinc<uint64_t><<<G, 256, 0, s>>>(out.rec.p, nc, k, out.vinc_off.p, cur.p,
                                              reinterpret_cast<uint64_t *>(out.vinc.p));
    else if (nc)
      k_fill_vinc<uint32_t><<<G, 256, 0, s>>>(out.rec.p, nc, k, out.vinc_off.p, cur.p, out.vinc.p);
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
}

}  // namespace cds
