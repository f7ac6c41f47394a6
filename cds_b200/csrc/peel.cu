// peel.cu -- (k,Psi)-clique-core decomposition and the density of every core.
//
// Replaces cliqueCoreDecompose (cudaCode/main.cu:252-343) with selectNodes /
// processNodesByWarp (cudaCode/src/helpers.cu:611-750), whose removal step
// scans every clique for each removed vertex, and the serial oracle's peel
// (cpuCode/c++/src/helpers.cpp:16-150), which removes one minimum-degree
// vertex at a time and records the density of what is left.
//
// Core numbers as the fixpoint of a local operator instead of a peel.  For
// a vertex v with clique set Psi(v), let x_C = min over the other members u
// of C of tau(u).  H(v) = the largest h with at least h cliques x_C >= h.
// Starting from tau = clique degree (an upper bound of the core number),
// tau(v) <- H(v), applied in any order, decreases monotonically and stops
// exactly at the clique-core numbers: a fixpoint F satisfies F <= core (the
// vertices with F >= h span at least h cliques each inside that set, so they
// lie in the h-core), and every iterate stays >= core (H is monotone and
// core is its fixpoint).  This is the local characterisation of nucleus
// decompositions (Sariyuce, Seshadhri, Pinar, VLDB 2018) for 1-vertex
// nuclei of k-cliques.  A sweep over all incidences is bulk-parallel work:
// the number of sweeps (about 30 on R-MAT graphs) replaces the number of
// peel levels (hundreds to thousands), each of which needs a grid-wide
// synchronisation.
//
// A sweep splits every vertex's incidence list into items of at most
// `chunk` incidences, one warp per item.  A vertex with one item gets an
// exact histogram of its x_C and its exact H, stored at once (later items of
// the sweep read it).  The items of a larger vertex (a hub) count x_C >=
// tau(v), the exact values tau-1 .. tau-32, and the rest in log-scale bins of
// sixteen per octave of the distance below that window, summed in global
// memory; the warp adding the last item computes the new value -- exact in
// the window, else the least upper bound the bins allow (still >= core, so
// the fixpoint is unchanged, and within about a seventeenth of the gap, which the
// next sweep refines).  A sweep in which no value changes saw every value in
// its final state, so it ends the loop.
//
// Densities: the alive set at each level of a peel is a core {v : core(v) >=
// L}; |V_L| and |Psi_L| (cliques whose smallest member core is >= L) come
// from two histograms and suffix sums, and the best level keeps the first
// (smallest) L with the largest |Psi_L| / |V_L|, as the level-by-level peel
// records it.  Instances of a batch (disjoint vertex ranges) are
// independent and share every sweep.
#include "device_util.cuh"
#include "stages.h"

#include <algorithm>
#include <cstdio>

namespace {

constexpr uint32_t UNSET = 0xFFFFFFFFu;
constexpr int WIN = 32;                       // exact values t-1 .. t-32 of a hub
constexpr int SUB_BITS = 4;
constexpr int SUB = 1 << SUB_BITS;            // bins per octave below them
constexpr int NLOG = 32 * SUB;                // log-scale bins below the window
constexpr int ACC_WORDS = 1 + WIN + NLOG;     // [0] count >= t, window, log bins
constexpr int MAX_CHUNK = 1024;               // incidences per item, at most
constexpr uint32_t MAX_READ_SWEEPS = 64;      // sweeps whose reads profiling records
constexpr int PACK_BITS = 21;                 // member id field of the packed layout
constexpr unsigned long long PACK_MASK = (1ull << PACK_BITS) - 1;
constexpr uint32_t PACK_MAX_N = 1u << PACK_BITS;  // vertices the packed layout can name

struct HParams {
  uint32_t n, k;
  const uint32_t *members;    // [m*k]
  const uint64_t *inc_off;    // [n+1]
  const uint32_t *inc;        // [k*m] clique ids, by vertex (clique layout)
  const unsigned long long *inc64;  // the same as u64 ids (2^32 or more cliques)
  const uint32_t *tup;        // [(k-1) * k*m] the other members, slot-major (member layout)
  const uint16_t *tup16;      // the same as 16-bit ids (graphs of at most 65,536 vertices)
  const unsigned long long *tup64;  // [k*m] the other members packed as 21-bit fields (k = 3, 4)
  uint64_t tup_stride;        // k*m
  uint32_t *tau;              // [n] upper bound of the core number
  const uint32_t *item_v;     // [nitems] vertex of each item
  const uint32_t *item_c;     // [nitems] its index among the vertex's items
  const uint32_t *vitems;     // [n] items of each vertex
  const uint64_t *nitems;     // items in all: item_off[n], on the device
  uint32_t chunk;             // a vertex with at most this many incidences is one item
  uint32_t warp_words;        // shared words per warp: max(chunk + 1, ACC_WORDS), rounded to 4
  uint32_t hub_chunk;         // incidences per item of a larger vertex (a hub)
  const uint32_t *big_slot;   // [n] slot of a vertex with several items
  const uint32_t *big_v;      // [nbig]
  uint32_t nbig;
  uint32_t *acc;              // [nbig * ACC_WORDS] counts of the current sweep
  uint32_t *big_done;         // [nbig] items counted in the current sweep
  uint32_t *ctl;              // [3 * 32] change flag, ~(smallest new value), by sweep mod 3
  const uint32_t *of_vertex;  // [n] instance of each vertex (null: one instance)
  uint32_t ninst;
  uint32_t *ichg;             // [3 * ninst] per-instance change flags, by sweep mod 3
  GridBarrier *bar;
  uint32_t *err;
  unsigned long long spin_limit;
  uint32_t max_sweeps;
  unsigned long long time_budget_ns;
  uint32_t *sweeps;           // sweeps run
  unsigned long long *reads;  // [MAX_READ_SWEEPS] incidences read per sweep (profiling; null: off)
  uint32_t static_pct;        // this percent of the items goes round-robin to the
                              // warps; the rest are taken from a per-sweep counter
};

template <bool CG>
__device__ __forceinline__ uint32_t ld_tau(const uint32_t *a) {
  return CG ? __ldcg(a) : *a;
}

// x_C for incidence i of vertex v: the smallest tau over the other members of
// its clique (CG: read at L2, never from a possibly older L1 copy).  TUP 1
// (2): the other members are stored per incidence as u32 (u16) ids, k-1
// coalesced streams; TUP 3: the k-1 <= 3 other members packed into one u64
// per incidence (21-bit ids); TUP 0 (4): the u32 (u64) clique id leads to
// its member record.
template <int K, int TUP, bool CG>
__device__ __forceinline__ uint32_t other_min(const HParams &p, uint64_t i, uint32_t v) {
  uint32_t x = UNSET;
  if (TUP == 3) {
    const unsigned long long q = __ldcs(p.tup64 + i);
#pragma unroll
    for (int j = 0; j < K - 1; j++) x = min(x, ld_tau<CG>(p.tau + (uint32_t)((q >> (PACK_BITS * j)) & PACK_MASK)));
    return x;
  }
  if (TUP == 1 || TUP == 2) {
#pragma unroll
    for (int j = 0; j < K - 1; j++) {
      const uint32_t w = TUP == 2 ? (uint32_t)__ldcs(p.tup16 + j * p.tup_stride + i)
                                  : __ldcs(p.tup + j * p.tup_stride + i);
      x = min(x, ld_tau<CG>(p.tau + w));
    }
    return x;
  }
  const uint64_t c = TUP == 4 ? (uint64_t)__ldg(p.inc64 + i) : (uint64_t)__ldg(p.inc + i);
  if (K == 4) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p.members) + c);
    const uint32_t a = q.x != v ? ld_tau<CG>(p.tau + q.x) : UNSET;
    const uint32_t b = q.y != v ? ld_tau<CG>(p.tau + q.y) : UNSET;
    const uint32_t d = q.z != v ? ld_tau<CG>(p.tau + q.z) : UNSET;
    const uint32_t e = q.w != v ? ld_tau<CG>(p.tau + q.w) : UNSET;
    x = min(min(a, b), min(d, e));
  } else if (K == 2) {
    const uint2 q = __ldg(reinterpret_cast<const uint2 *>(p.members) + c);
    x = ld_tau<CG>(p.tau + (q.x != v ? q.x : q.y));
  } else {
    const uint32_t k = K ? K : p.k;
    const uint32_t *mc = p.members + (uint64_t)c * k;
#pragma unroll 4
    for (uint32_t j = 0; j < k; j++) {
      const uint32_t w = __ldg(mc + j);
      if (w != v) x = min(x, ld_tau<CG>(p.tau + w));
    }
  }
  return x;
}

// x_C of incidences i, i+32, ..., i+32(U-1) (those below e; UNSET for the
// rest), with every load of the U incidences issued before any is used
constexpr int UNROLL = 4;
template <int K, int TUP, bool CG>
__device__ __forceinline__ void other_min_x4(const HParams &p, uint64_t i, uint64_t e, uint32_t v,
                                             uint32_t (&x)[UNROLL]) {
  if (TUP == 3) {
    unsigned long long q[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; u++) q[u] = i + 32u * u < e ? __ldcs(p.tup64 + i + 32u * u) : 0ull;
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      x[u] = UNSET;
      if (i + 32u * u < e) {
#pragma unroll
        for (int j = 0; j < K - 1; j++)
          x[u] = min(x[u], ld_tau<CG>(p.tau + (uint32_t)((q[u] >> (PACK_BITS * j)) & PACK_MASK)));
      }
    }
  } else if (TUP == 1 || TUP == 2) {
    constexpr int KM = K > 1 ? K - 1 : 1;
    uint32_t w[UNROLL][KM];
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      const uint64_t iu = i + 32u * u;
#pragma unroll
      for (int j = 0; j < KM; j++)
        w[u][j] = iu >= e ? 0u
                  : TUP == 2 ? (uint32_t)__ldcs(p.tup16 + j * p.tup_stride + iu)
                             : __ldcs(p.tup + j * p.tup_stride + iu);
    }
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      x[u] = UNSET;
      if (i + 32u * u < e) {
#pragma unroll
        for (int j = 0; j < KM; j++) x[u] = min(x[u], ld_tau<CG>(p.tau + w[u][j]));
      }
    }
  } else {
#pragma unroll
    for (int u = 0; u < UNROLL; u++)
      x[u] = i + 32u * u < e ? other_min<K, TUP, CG>(p, i + 32u * u, v) : UNSET;
  }
}

// An item's packed member tuples [b, e) brought from DRAM into L2 ahead of
// its loads by one bulk prefetch (16-byte aligned: b rounded down and e up to
// even; the array holds one spare element past its end).  The sweep's loads
// then meet L2 latency after the first window instead of DRAM latency for
// every window, with no register or shared memory held for it.
__device__ __forceinline__ void prefetch_tuples(const unsigned long long *tup64, uint64_t b, uint64_t e) {
  const uint64_t b0 = b & ~1ull, e0 = (e + 1) & ~1ull;
  if (e0 > b0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(tup64 + b0), "r"((uint32_t)((e0 - b0) * 8))
                 : "memory");
}

// Exact histogram of one single-item vertex: hist[min(x_C, t)] += 1 over
// its incidences; returns H exactly.  hist has t+1 <= chunk+1 words.
template <int K, int TUP, bool CG>
__device__ __forceinline__ uint32_t h_exact(const HParams &p, uint32_t v, uint32_t t, uint64_t b,
                                            uint64_t e, uint32_t *hist, uint64_t &read) {
  const uint32_t lane = lane_id();
  for (uint32_t i = lane; i <= t; i += 32) hist[i] = 0;
  __syncwarp();
  // x >= t (most cliques of a vertex at its fixpoint) is counted in a
  // register: as a shared-memory atomic every lane would hit hist[t]
  uint32_t ge = 0;
  for (uint64_t i0 = b; i0 < e; i0 += 32 * UNROLL) {
    const uint64_t i = i0 + lane;
    uint32_t x[UNROLL];
    other_min_x4<K, TUP, CG>(p, i, e, v, x);
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      if (i + 32u * u >= e) continue;
      if (x[u] >= t) ge++;
      else atomicAdd(&hist[x[u]], 1u);
    }
    // t cliques with x >= t already give H >= t, and H <= t: the value
    // stands, and the rest of the list cannot change that
    if (__reduce_add_sync(CDS_FULL, ge) >= t) {
      __syncwarp();
      read += min(e, i0 + 32 * UNROLL) - b;
      return t;
    }
  }
  read += e - b;
  ge = __reduce_add_sync(CDS_FULL, ge);
  __syncwarp();
  if (lane == 0) hist[t] += ge;
  __syncwarp();
  // largest h with (values >= h) >= h, 32 candidates at a time from the top;
  // h = 0 always qualifies, so the loop ends by top = 31 at the latest
  uint32_t acc = 0;
  for (int top = (int)t;; top -= 32) {
    const int h = top - (int)lane;
    const uint32_t c = h >= 0 ? hist[h] : 0u;
    const uint32_t incl = warp_inclusive_scan(c);
    const bool ok = h <= 0 || acc + incl >= (uint32_t)h;
    const uint32_t m = __ballot_sync(CDS_FULL, ok);
    if (m) {
      __syncwarp();
      return (uint32_t)(top - (__ffs(m) - 1));
    }
    acc += __shfl_sync(CDS_FULL, incl, 31);
  }
}

// Log-scale bin of a distance e = t-WIN-x >= 1 below the window: octave j =
// floor(log2 e) split into SUB = 16 parts by the four bits after the
// leading one, so bin (j, s) holds e in [ceil((16+s) 2^j / 16),
// ceil((17+s) 2^j / 16)) (empty for some s when j < 4).  Bins grow with e.
__device__ __forceinline__ uint32_t log_bin(uint32_t e) {
  const uint32_t j = 31 - __clz(e);
  const uint32_t s = j >= SUB_BITS ? (e >> (j - SUB_BITS)) & (SUB - 1u) : (e << (SUB_BITS - j)) & (SUB - 1u);
  return j * SUB + s;
}
__device__ __forceinline__ unsigned long long log_bin_lo(uint32_t b) {  // smallest e of bin b
  return (((unsigned long long)(SUB + b % SUB) << (b / SUB)) + SUB - 1) >> SUB_BITS;
}

// Counts of one item of a hub (t fixed for the sweep): [0] x >= t,
// [1 + d] x = t-1-d for d < WIN, [1 + WIN + log_bin(t-WIN-x)] x < t-WIN.
template <int K, int TUP, bool CG>
__device__ __forceinline__ void hub_counts(const HParams &p, uint32_t v, uint32_t t, uint64_t b,
                                           uint64_t e, uint32_t *cnt) {
  const uint32_t lane = lane_id();
  for (uint32_t i = lane; i < ACC_WORDS; i += 32) cnt[i] = 0;
  __syncwarp();
  uint32_t ge = 0;
  for (uint64_t i = b + lane; i < e; i += 32 * UNROLL) {
    uint32_t x[UNROLL];
    other_min_x4<K, TUP, CG>(p, i, e, v, x);
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      if (i + 32u * u >= e) continue;
      if (x[u] >= t) {
        ge++;
      } else {
        const uint32_t d = t - 1u - x[u];
        atomicAdd(&cnt[d < WIN ? 1 + d : 1 + WIN + log_bin(d + 1u - WIN)], 1u);
      }
    }
  }
  ge = __reduce_add_sync(CDS_FULL, ge);
  __syncwarp();
  if (lane == 0) cnt[0] = ge;
  __syncwarp();
}

// New value of a hub from its summed counts: H exactly when it lies in the
// window, else the least upper bound the log bins give (H < t - WIN there):
// the top value of the first bin, from the top, whose lowest value h has
// at least h counts at or above it -- every h above it fails -- so that a
// drop far below the window shrinks the gap about seventeenfold per sweep.
__device__ __forceinline__ uint32_t hub_tau(uint32_t t, const uint32_t *acc) {
  const uint32_t lane = lane_id();
  const uint32_t ge = __ldcg(acc);
  if (ge >= t) return t;
  // window: lane d checks h = t-1-d
  const uint32_t wi = warp_inclusive_scan(__ldcg(acc + 1 + lane));
  const long long h = (long long)t - 1 - lane;
  uint32_t m = __ballot_sync(CDS_FULL, h <= 0 || (long long)ge + wi >= h);
  if (m) return (uint32_t)(t - 1 - (__ffs(m) - 1));
  // below the window, 32 bins at a time; bin (j, s) holds x in
  // [t-WIN-hi+1, t-WIN-lo] for its e range [lo, hi).  The last bins reach
  // x <= 0, so some bin qualifies.
  unsigned long long base = (unsigned long long)ge + __shfl_sync(CDS_FULL, wi, 31);
  for (uint32_t b0 = 0; b0 < NLOG; b0 += 32) {
    const uint32_t b = b0 + lane;
    const uint32_t cnt = __ldcg(acc + 1 + WIN + b);
    const unsigned long long incl = base + warp_inclusive_scan(cnt);
    const unsigned long long lo = log_bin_lo(b), hi = log_bin_lo(b + 1);  // bin NLOG starts at 2^32
    const long long xlo = (long long)t - WIN - (long long)hi + 1;
    const bool ok = hi > lo && (xlo <= 0 || (long long)incl >= xlo);
    m = __ballot_sync(CDS_FULL, ok);
    if (m) {
      const uint32_t bb = b0 + (__ffs(m) - 1);
      const long long xhi = (long long)t - WIN - (long long)log_bin_lo(bb);
      return xhi > 0 ? (uint32_t)xhi : 0u;
    }
    base = __shfl_sync(CDS_FULL, incl, 31);
  }
  return 0;  // not reached: the last bin reaches x <= 0
}

template <int K, int TUP>
__global__ void __launch_bounds__(512, 2) k_hindex(HParams p) {
  extern __shared__ uint32_t s_hist[];
  __shared__ uint32_t s_any, s_low;  // per-sweep block summary of changes
  uint32_t *hist = s_hist + (threadIdx.x >> 5) * p.warp_words;
  if (threadIdx.x == 0) {
    s_any = 0;
    s_low = 0;
  }
  __syncthreads();
  const uint32_t lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  const unsigned long long t0 = globaltimer_ns();
  const uint32_t nitems = (uint32_t)*p.nitems;
  uint32_t it = 0;
  // After a sweep without change, one more reads every value at L2: only a
  // sweep that saw the current values and changed nothing ends the loop.
  bool verify = false;
  for (; it < p.max_sweeps; it++) {
    uint32_t *changed = p.ctl + (it % 3) * 32;
    uint32_t *ichg = p.ichg + (it % 3) * p.ninst;
    // an instance none of whose values changed in the last sweep is at its
    // fixpoint (its vertices read only its own values): skip it, except in
    // a verifying sweep
    const uint32_t *quiet_src = it > 0 && !verify ? p.ichg + ((it + 2) % 3) * p.ninst : nullptr;
    if (leader) {
      // slot (it+1)%3 was last read right after the barrier of sweep it-2,
      // before every block passed the barrier of sweep it-1
      p.ctl[((it + 1) % 3) * 32] = 0;
      p.ctl[((it + 1) % 3) * 32 + 2] = 0;
      p.ctl[((it + 1) % 3) * 32 + 3] = 0;  // the item counter of that sweep
      if (globaltimer_ns() - t0 > p.time_budget_ns) atomicOr(p.err, DEV_ERR_TIMEOUT);
    }
    if (blockIdx.x == 0)  // the per-instance flags of slot (it+1)%3 likewise
      for (uint32_t i = threadIdx.x; i < p.ninst; i += blockDim.x) p.ichg[((it + 1) % 3) * p.ninst + i] = 0;
    bool any = false;
    // Every value that changed in the last sweep ended at or above `low`
    // (slot word 2 holds ~min, so zero means none).  A vertex with tau < low
    // reads each clique through min(x_C, tau), which those changes cannot
    // move (old and new values are both >= tau), and it did not change
    // itself (its value would be >= low), so its value is still exact: skip
    // it.  The verifying sweep recounts everything.
    const uint32_t low = it > 0 && !verify ? ~*(volatile uint32_t *)(p.ctl + ((it + 2) % 3) * 32 + 2) : 0u;
    uint32_t wmin = UNSET;  // smallest new value this warp stored
    uint64_t wread = 0;     // incidences this warp read (profiling)
    // items in the static part go to the warps round-robin; then each warp
    // takes the next item of the tail from the sweep's counter (early exits
    // make item costs uneven, and a warp left idle waits at the barrier)
    const uint32_t stat = (uint32_t)((uint64_t)nitems * p.static_pct / 100u);
    uint32_t *tail = p.ctl + (it % 3) * 32 + 3;
    auto next_tail = [&]() -> uint32_t {
      uint32_t got = 0;
      if (lane == 0) got = atomicAdd(tail, 1u);
      return stat + __shfl_sync(CDS_FULL, got, 0);
    };
    for (uint32_t r = gwarp < stat ? gwarp : next_tail(); r < nitems;
         r = r + nwarps < stat ? r + nwarps : next_tail()) {
      const uint32_t v = p.item_v[r];
      // the vertex's own value at L2: every item of a hub must count against
      // the same t, and an L1 line filled before another SM stored the
      // hub's new value would give an older one
      const uint32_t t = __ldcg(p.tau + v);
      if (t < low || t == 0) continue;
      const uint32_t inst = p.of_vertex ? p.of_vertex[v] : 0u;
      if (quiet_src && !__ldcg(quiet_src + inst)) continue;
      const uint32_t nit = p.vitems[v];
      const uint64_t ib = p.inc_off[v], ie = p.inc_off[v + 1];
      const bool hub = ie - ib > p.chunk;
      const uint32_t len = hub ? p.hub_chunk : p.chunk;
      const uint64_t b = ib + (uint64_t)p.item_c[r] * len;
      const uint64_t e = min(b + len, ie);
      uint32_t nt = t;
      if (!hub) {
        // the whole list (t <= clique degree <= chunk): exact, and visible
        // to the rest of the sweep at once
        if (TUP == 3 && lane == 0) prefetch_tuples(p.tup64, b, e);
        nt = verify ? h_exact<K, TUP, true>(p, v, t, b, e, hist, wread)
                    : h_exact<K, TUP, false>(p, v, t, b, e, hist, wread);
      } else {
        // a hub: add this item's counts; the warp adding the last item
        // computes the new value, so it too is visible within the sweep,
        // and no item of the hub reads its value after that
        const uint32_t bi = p.big_slot[v];
        uint32_t *a = p.acc + (uint64_t)bi * ACC_WORDS;
        // items that finished earlier in this sweep may already have found
        // t cliques with x >= t: then H = t whatever this item holds, and
        // it only reports that it is done
        const uint32_t have = __shfl_sync(CDS_FULL, lane == 0 ? __ldcg(a) : 0u, 0);
        if (have < t) {
          if (TUP == 3 && lane == 0) prefetch_tuples(p.tup64, b, e);
          if (verify) hub_counts<K, TUP, true>(p, v, t, b, e, hist);
          else hub_counts<K, TUP, false>(p, v, t, b, e, hist);
          wread += e - b;
          for (uint32_t i = lane; i < ACC_WORDS; i += 32)
            if (hist[i]) atomicAdd(a + i, hist[i]);
        }
        __syncwarp();
        uint32_t prev = 0;
        if (lane == 0) {
          __threadfence();  // the counts above, then the item's completion
          prev = atomicAdd(p.big_done + bi, 1u);
          if (prev + 1 == nit) __threadfence();  // the last item's reader sees every count
        }
        prev = __shfl_sync(CDS_FULL, prev, 0);
        __syncwarp();
        if (prev + 1 < nit) continue;
        nt = hub_tau(t, a);
        __syncwarp();
        for (uint32_t i = lane; i < ACC_WORDS; i += 32) a[i] = 0;
        if (lane == 0) p.big_done[bi] = 0;
      }
      if (nt < t) {
        if (lane == 0) {
          p.tau[v] = nt;
          ichg[inst] = 1;
        }
        any = true;
        wmin = min(wmin, nt);
      }
    }
    if (p.reads && lane == 0 && wread && it < MAX_READ_SWEEPS) atomicAdd(p.reads + it, (unsigned long long)wread);
    // the block's change flag and smallest new value, then one global update
    if (any && lane == 0) {
      s_any = 1;
      atomicMax(&s_low, ~wmin);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_any) {
      changed[0] = 1;
      atomicMax(changed + 2, s_low);
      s_any = 0;  // read again only after the next sweep's items
      s_low = 0;
    }
    if (!grid_sync(p.bar, p.err, p.spin_limit)) break;
    if (*(volatile uint32_t *)changed == 0) {
      if (verify) {
        it++;
        break;
      }
      verify = true;
    } else {
      verify = false;
    }
  }
  if (leader) {
    *p.sweeps = it;
    if (it >= p.max_sweeps) atomicOr(p.err, DEV_ERR_TIMEOUT);
  }
}

// incidence lists: slot j of clique c goes to members[c*k+j]'s list (ids
// as u32, or as u64 when there are 2^32 or more cliques)
template <typename I>
__global__ void k_fill_incidence(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                                 const uint64_t *__restrict__ inc_off, uint32_t *__restrict__ cursor,
                                 I *__restrict__ inc) {
  const uint64_t total = m * k;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
    const uint64_t t = base + threadIdx.x;
    // slot-major order: lanes see the same slot of consecutive cliques, which
    // share their root, so the cursor atomics aggregate
    const bool ok = t < total;
    uint32_t v = UNSET;
    uint64_t c = 0;
    if (ok) {
      const uint64_t j = t / m;
      c = t - j * m;
      v = members[c * k + j];
    }
    const uint32_t grp = __match_any_sync(CDS_FULL, v);
    const uint32_t leader = __ffs(grp) - 1;
    uint32_t at = 0;
    if (ok && leader == lane_id()) at = atomicAdd(&cursor[v], (uint32_t)__popc(grp));
    at = __shfl_sync(grp, at, leader);
    if (ok) inc[inc_off[v] + at + __popc(grp & ((1u << lane_id()) - 1u))] = (I)c;
  }
}

// member layout: incidence (v, c) stores the k-1 other members of c, in
// slot order, in k-1 arrays of k*m entries
template <typename T>
__global__ void k_fill_tuples(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                              const uint64_t *__restrict__ inc_off, uint32_t *__restrict__ cursor,
                              T *__restrict__ tup) {
  const uint64_t total = m * k;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
    const uint64_t t = base + threadIdx.x;
    const bool ok = t < total;
    uint32_t v = UNSET, j = 0;
    uint64_t c = 0;
    if (ok) {
      j = (uint32_t)(t / m);
      c = t - (uint64_t)j * m;
      v = members[c * k + j];
    }
    const uint32_t grp = __match_any_sync(CDS_FULL, v);
    const uint32_t leader = __ffs(grp) - 1;
    uint32_t at = 0;
    if (ok && leader == lane_id()) at = atomicAdd(&cursor[v], (uint32_t)__popc(grp));
    at = __shfl_sync(grp, at, leader);
    if (ok) {
      const uint64_t pos = inc_off[v] + at + __popc(grp & ((1u << lane_id()) - 1u));
      for (uint32_t s = 0; s + 1 < k; s++) tup[s * total + pos] = (T)members[c * k + (s < j ? s : s + 1)];
    }
  }
}

// packed member layout: incidence (v, c) stores the k-1 <= 3 other members
// of c, in slot order, as 21-bit fields of one u64
__global__ void k_fill_tuples64(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                                const uint64_t *__restrict__ inc_off, uint32_t *__restrict__ cursor,
                                unsigned long long *__restrict__ tup) {
  // clique-major: a thread reads its clique's record once and places the k
  // incidences, one warp-aggregated cursor round per slot (consecutive
  // records share their root and, in runs, their next members)
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < m; base += stride) {
    const uint64_t c = base + threadIdx.x;
    const bool ok = c < m;
    uint32_t mem[4] = {UNSET, UNSET, UNSET, UNSET};
    if (ok) {
      if (k == 4) {
        const uint4 r = *reinterpret_cast<const uint4 *>(members + c * 4);
        mem[0] = r.x;
        mem[1] = r.y;
        mem[2] = r.z;
        mem[3] = r.w;
      } else {
        for (uint32_t j = 0; j < k; j++) mem[j] = members[c * k + j];
      }
    }
    // every slot's cursor atomic and list offset are issued before any is
    // used: the k round trips to L2 overlap instead of following each other
    uint32_t grp[4], at[4];
    uint64_t off[4];
#pragma unroll
    for (uint32_t j = 0; j < 4; j++) {
      grp[j] = 0;
      at[j] = 0;
      off[j] = 0;
      if (j >= k) continue;
      const uint32_t v = ok ? mem[j] : UNSET;
      grp[j] = __match_any_sync(CDS_FULL, v);
      if (ok && __ffs(grp[j]) - 1 == (int)lane_id()) at[j] = atomicAdd(&cursor[v], (uint32_t)__popc(grp[j]));
      if (ok) off[j] = inc_off[v];
    }
#pragma unroll
    for (uint32_t j = 0; j < 4; j++) {
      if (j >= k) continue;
      const uint32_t leader = __ffs(grp[j]) - 1;
      const uint32_t base = __shfl_sync(grp[j], at[j], leader);
      if (ok) {
        const uint64_t pos = off[j] + base + __popc(grp[j] & ((1u << lane_id()) - 1u));
        unsigned long long q = 0;
        uint32_t f = 0;
#pragma unroll
        for (uint32_t s2 = 0; s2 < 4; s2++)
          if (s2 < k && s2 != j) q |= (unsigned long long)mem[s2] << (PACK_BITS * f++);
        tup[pos] = q;
      }
    }
  }
}

// items of each vertex: one up to `chunk` incidences (an exact histogram in
// shared memory), else ceil(clique degree / hub_chunk) hub items
__global__ void k_item_count(const uint32_t *__restrict__ cdeg, uint32_t n, uint32_t chunk,
                             uint32_t hub_chunk, uint32_t *__restrict__ items,
                             uint32_t *__restrict__ multi) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t d = cdeg[v];
    const bool hub = d > chunk;
    items[v] = hub ? (d + hub_chunk - 1) / hub_chunk : (d ? 1u : 0u);
    multi[v] = hub ? 1u : 0u;
  }
}

// Item order.  With `peel_order` set, vertices go in ascending classes of
// clique degree (powers of two): a single-item vertex's new value is visible
// to the rest of the sweep, so low-degree vertices settle first and the hubs,
// counted last, read fresher values.  Otherwise items follow vertex ids.
// bcur[32] counts, then places, the vertices of each class.
__global__ void k_class_count(const uint32_t *__restrict__ cdeg, uint32_t n, uint32_t *__restrict__ bcur) {
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t v = base + threadIdx.x;
    const uint32_t d = v < n ? cdeg[v] : 0u;
    agg_add_u32(bcur, d ? 31u - __clz(d) : 0u, d != 0);
  }
}
__global__ void k_class_scan(uint32_t *bcur) {  // one warp: exclusive scan of the 32 counts
  const uint32_t x = bcur[lane_id()];
  bcur[lane_id()] = warp_inclusive_scan(x) - x;
}
__global__ void k_class_place(const uint32_t *__restrict__ cdeg, const uint32_t *__restrict__ items,
                              uint32_t n, uint32_t *__restrict__ bcur, uint32_t *__restrict__ perm,
                              uint32_t *__restrict__ pitems) {
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t v = base + threadIdx.x;
    const uint32_t d = v < n ? cdeg[v] : 0u;
    const uint32_t at = agg_inc(bcur, d ? 31u - __clz(d) : 0u, d != 0);
    if (d) {
      perm[at] = v;
      pitems[at] = items[v];
    }
  }
}

// item_v / item_c of the vertices in order (perm null: ids, n of them; else
// the bcur[31] placed ones), and each hub's accumulator slot
__global__ void k_item_fill(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ nplaced,
                            const uint64_t *__restrict__ item_off, const uint64_t *__restrict__ big_off,
                            uint32_t n, uint32_t *__restrict__ item_v, uint32_t *__restrict__ item_c,
                            uint32_t *__restrict__ big_slot, uint32_t *__restrict__ big_v) {
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t np = perm ? nplaced[31] : n;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < np; i += warps) {
    const uint32_t v = perm ? perm[i] : i;
    const uint64_t b = item_off[i], e = item_off[i + 1];
    for (uint64_t r = b + lane_id(); r < e; r += 32) {
      item_v[r] = v;
      item_c[r] = (uint32_t)(r - b);
    }
  }
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps)
    if (lane_id() == 0) {
      const bool multi = big_off[v + 1] > big_off[v];
      big_slot[v] = multi ? (uint32_t)big_off[v] : UNSET;
      if (multi) big_v[big_off[v]] = v;
    }
}

// largest core per instance and the vertex histogram of core numbers
__global__ void k_inst_maxcore(const uint32_t *__restrict__ core, uint32_t n,
                               const uint32_t *__restrict__ of_vertex, uint32_t *__restrict__ out) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint32_t v = base + threadIdx.x;
    const bool ok = v < n;
    const uint32_t key = ok ? (of_vertex ? of_vertex[v] : 0u) : UNSET;
    const uint32_t grp = __match_any_sync(CDS_FULL, key);
    const uint32_t m = __reduce_max_sync(grp, ok ? core[v] : 0u);
    if (ok && (__ffs(grp) - 1) == (int)lane_id()) atomicMax(out + key, m);
  }
}

// hv[hoff[i] + L] = vertices of instance i with core L; hc likewise for
// cliques by their smallest member core
__global__ void k_core_hist(const uint32_t *__restrict__ core, uint32_t n,
                            const uint32_t *__restrict__ of_vertex,
                            const uint64_t *__restrict__ hoff, unsigned long long *__restrict__ hv) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint32_t v = base + threadIdx.x;
    const bool ok = v < n;
    uint64_t key = ~0ull;
    if (ok) key = hoff[of_vertex ? of_vertex[v] : 0u] + core[v];
    const uint32_t grp = __match_any_sync(CDS_FULL, key);
    if (ok && (__ffs(grp) - 1) == (int)lane_id()) atomicAdd(hv + key, (unsigned long long)__popc(grp));
  }
}

// (cmin[c] = that smallest member core: the densest-core stage derives its
// clique flags from it without reading the records again)
__global__ void k_clique_hist(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                              const uint32_t *__restrict__ core, const uint32_t *__restrict__ of_vertex,
                              const uint64_t *__restrict__ hoff, unsigned long long *__restrict__ hc,
                              uint32_t *__restrict__ cmin) {
  // A warp whose 32 cliques share one level (the cliques inside a dense
  // core) adds to a count its lane 0 keeps while the level stays the same,
  // instead of an atomic per step on that level's word.
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t wkey = ~0ull;
  unsigned long long wn = 0;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < m; base += stride) {
    const uint64_t c = base + threadIdx.x;
    const bool ok = c < m;
    uint64_t key = ~0ull;
    if (ok) {
      const uint32_t *mc = members + c * k;
      uint32_t lo = UNSET, first;
      if (k == 4) {  // the record in one 16-byte load
        const uint4 q = *reinterpret_cast<const uint4 *>(mc);
        lo = min(min(core[q.x], core[q.y]), min(core[q.z], core[q.w]));
        first = q.x;
      } else {
        for (uint32_t j = 0; j < k; j++) lo = min(lo, core[mc[j]]);
        first = mc[0];
      }
      cmin[c] = lo;
      key = hoff[of_vertex ? of_vertex[first] : 0u] + lo;
    }
    const uint64_t k0 = __shfl_sync(CDS_FULL, key, 0);
    if (__all_sync(CDS_FULL, ok && key == k0)) {
      if (lane_id() == 0) {
        if (k0 != wkey) {
          if (wn) atomicAdd(hc + wkey, wn);
          wkey = k0;
          wn = 0;
        }
        wn += 32;
      }
      continue;
    }
    const uint32_t grp = __match_any_sync(CDS_FULL, key);
    if (ok && (__ffs(grp) - 1) == (int)lane_id()) atomicAdd(hc + key, (unsigned long long)__popc(grp));
  }
  if (lane_id() == 0 && wn) atomicAdd(hc + wkey, wn);
}

// One block per instance: suffix sums over L of both histograms give the
// core {core >= L}; keep the smallest L of largest density (the first level
// a peel would record), and count the distinct core numbers.
__global__ void __launch_bounds__(512) k_best_level(const uint64_t *__restrict__ hoff,
                                                    const unsigned long long *__restrict__ hv,
                                                    const unsigned long long *__restrict__ hc,
                                                    uint32_t ninst, unsigned long long *__restrict__ best_num,
                                                    unsigned long long *__restrict__ best_den,
                                                    uint32_t *__restrict__ levels,
                                                    uint32_t *__restrict__ best_lvl) {
  __shared__ unsigned long long s_v, s_c;
  __shared__ unsigned long long s_bn[16], s_bd[16];
  __shared__ uint32_t s_lv[16], s_bl[16];
  for (uint32_t i = blockIdx.x; i < ninst; i += gridDim.x) {
    const uint64_t b = hoff[i], nb = hoff[i + 1] - b;
    if (threadIdx.x == 0) {
      s_v = 0;
      s_c = 0;
    }
    __syncthreads();
    unsigned long long bn = 0, bd = 0;
    uint32_t lv = 0, bl = 0;  // bl: the level of (bn, bd)
    // chunks of blockDim * LEVEL_ITEMS bins from the top (largest L) down;
    // thread t holds LEVEL_ITEMS consecutive bins below those of thread t-1
    constexpr int LEVEL_ITEMS = 8;
    for (uint64_t top = nb; top > 0;) {
      const uint64_t span = (uint64_t)blockDim.x * LEVEL_ITEMS;
      const uint64_t lo = top > span ? top - span : 0;
      const uint64_t first = top - 1 - (uint64_t)threadIdx.x * LEVEL_ITEMS;  // this thread's top bin
      unsigned long long xv[LEVEL_ITEMS], xc[LEVEL_ITEMS], tv = 0, tc = 0;
#pragma unroll
      for (int j = 0; j < LEVEL_ITEMS; j++) {
        const uint64_t L = first - j;
        const bool in = (uint64_t)threadIdx.x * LEVEL_ITEMS + j < top - lo;  // L in [lo, top)
        xv[j] = in ? hv[b + L] : 0;
        xc[j] = in ? hc[b + L] : 0;
        tv += xv[j];
        tc += xc[j];
      }
      unsigned long long chunk_v, chunk_c;
      // suffix sums above this thread's first bin
      unsigned long long sv = block_exclusive_scan<unsigned long long>(tv, &chunk_v) + s_v;
      unsigned long long sc = block_exclusive_scan<unsigned long long>(tc, &chunk_c) + s_c;
#pragma unroll
      for (int j = 0; j < LEVEL_ITEMS; j++) {
        sv += xv[j];
        sc += xc[j];
        if (xv[j]) {  // a level with vertices (bins outside [lo, top) hold 0)
          lv++;
          // sc/sv > bn/bd, or equal with a smaller L (later in this loop)
          const unsigned long long lh = __umul64hi(sc, bd), ll = sc * bd;
          const unsigned long long rh = __umul64hi(bn, sv), rl = bn * sv;
          if (bd == 0 || lh > rh || (lh == rh && ll >= rl)) {
            bn = sc;
            bd = sv;
            bl = (uint32_t)(first - j);
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s_v += chunk_v;
        s_c += chunk_c;
      }
      __syncthreads();
      top = lo;
    }
    // the block's best: largest density, then smallest L; every thread's
    // candidate has the smallest L among its ties, and L falls with the
    // thread's progress, so among equal densities the larger sv wins
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long on = __shfl_down_sync(CDS_FULL, bn, o);
      const unsigned long long od = __shfl_down_sync(CDS_FULL, bd, o);
      const uint32_t ol = __shfl_down_sync(CDS_FULL, bl, o);
      lv += __shfl_down_sync(CDS_FULL, lv, o);
      if (od) {
        const unsigned long long lh = __umul64hi(on, bd), ll = on * bd;
        const unsigned long long rh = __umul64hi(bn, od), rl = bn * od;
        const bool gt = lh > rh || (lh == rh && ll > rl);
        const bool eq = lh == rh && ll == rl;
        if (bd == 0 || gt || (eq && od > bd)) {
          bn = on;
          bd = od;
          bl = ol;
        }
      }
    }
    if (lane_id() == 0) {
      s_bn[threadIdx.x >> 5] = bn;
      s_bd[threadIdx.x >> 5] = bd;
      s_lv[threadIdx.x >> 5] = lv;
      s_bl[threadIdx.x >> 5] = bl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long fn = 0, fd = 0;
      uint32_t fl = 0, fb = 0;
      for (uint32_t w = 0; w < (blockDim.x >> 5); w++) {
        fl += s_lv[w];
        const unsigned long long on = s_bn[w], od = s_bd[w];
        if (!od) continue;
        const unsigned long long lh = __umul64hi(on, fd), ll = on * fd;
        const unsigned long long rh = __umul64hi(fn, od), rl = fn * od;
        const bool gt = lh > rh || (lh == rh && ll > rl);
        const bool eq = lh == rh && ll == rl;
        if (fd == 0 || gt || (eq && od > fd)) {
          fn = on;
          fd = od;
          fb = s_bl[w];
        }
      }
      best_num[i] = fn;
      best_den[i] = fd;
      levels[i] = fl;
      best_lvl[i] = fb;
    }
    __syncthreads();
  }
}

}  // namespace

namespace cds {

void peel(cds_ctx *c, cudaStream_t s, uint32_t n, const Cliques &cl, const Instances &inst,
          const Tuning &t, uint32_t gl_buffer_size, PeelOut &out) {
  const uint32_t k = cl.k;
  const uint64_t m = cl.count;
  const uint32_t ninst = inst.count;
  const uint32_t *of_vertex = ninst > 1 ? inst.of_vertex.p : nullptr;
  out.core.c = c;
  out.core.s = s;
  out.core.alloc(n + 1);
  out.best_num.assign(ninst, 0);
  out.best_den.assign(ninst, 0);
  out.inst_max_core.assign(ninst, 0);
  out.inst_levels.assign(ninst, 0);
  out.best_level.assign(ninst, 0);
  out.levels = 0;
  out.max_core = 0;
  if (n == 0) return;

  // vertex -> clique incidence CSR: for k <= 4 the other members of each
  // incidence (streamed by every sweep), falling back to clique ids (one
  // member record gathered per incidence) when that does not fit the budget
  DBuf<uint64_t> inc_off(c, s, n + 1);
  scan_u32(cl.cdeg.p, inc_off.p, n, c, s);
  DBuf<uint32_t> inc, tup;
  DBuf<uint16_t> tup16;
  DBuf<unsigned long long> tup64, inc64;
  inc.c = tup.c = tup16.c = tup64.c = inc64.c = c;
  inc.s = tup.s = tup16.s = tup64.s = inc64.s = s;
  // clique ids past 32 bits: 2^32 or more cliques (or the flag that forces
  // that layout); the member layouts below need no clique ids at all
  const bool wide_ids = m >= 0xFFFFFFFFull || (c->flags & CDS_CONFIG_WIDE_CLIQUE_IDS);
  bool tuple = false;
  const bool narrow = n <= 65536;  // member ids fit 16 bits
  // k = 3, 4 above that: the other members packed into one u64 (8 bytes an
  // incidence instead of 4(k-1)), while ids fit 21 bits
  const bool packed = !narrow && (k == 3 || k == 4) && n <= PACK_MAX_N;
  if (k <= 4 && m && !(c->flags & (CDS_CONFIG_COMPACT_PEEL | CDS_CONFIG_WIDE_CLIQUE_IDS))) {
    try {
      if (narrow) tup16.alloc(m * k * (k - 1) + 1);
      else if (packed) tup64.alloc(m * k + 1);
      else tup.alloc(m * k * (k - 1) + 1);
      tuple = true;
    } catch (const Error &e) {
      if (e.status != CDS_ERR_OOM) throw;
    }
  }
  if (!tuple && wide_ids) inc64.alloc(m * k + 1);
  else if (!tuple) inc.alloc(m * k + 1);
  {
    DBuf<uint32_t> cursor(c, s, n);
    cursor.zero();
    if (m) {
      ProfScope ps(c, s, "peel_incidence");
      if (tuple && narrow)
        k_fill_tuples<uint16_t><<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p, cursor.p,
                                                                tup16.p);
      else if (tuple && packed)
        k_fill_tuples64<<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p, cursor.p, tup64.p);
      else if (tuple)
        k_fill_tuples<uint32_t><<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p, cursor.p,
                                                                tup.p);
      else if (wide_ids)
        k_fill_incidence<unsigned long long><<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p,
                                                                            cursor.p, inc64.p);
      else
        k_fill_incidence<uint32_t><<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p, cursor.p,
                                                                  inc.p);
      count_launch();
      CDS_CUDA(cudaGetLastError());
    }
  }

  // Work items of at most `chunk` incidences; the reference's glBufferSize
  // (a per-block removal buffer length) has no counterpart here.
  (void)gl_buffer_size;
  const uint32_t chunk = (uint32_t)std::max(64, std::min(t.peel_chunk, MAX_CHUNK));
  DBuf<uint32_t> items(c, s, n), multi(c, s, n);
  const uint32_t hub_chunk = chunk;  // larger hub items save flushes but cost sweeps
  k_item_count<<<c->sm_count * 4, 256, 0, s>>>(cl.cdeg.p, n, chunk, hub_chunk, items.p, multi.p);
  count_launch();
  // item order: by ascending degree class (t.peel_order) or by vertex id
  DBuf<uint32_t> bcur(c, s, 32), perm, pitems;
  perm.c = pitems.c = c;
  perm.s = pitems.s = s;
  if (t.peel_order) {
    perm.alloc(n + 1);
    pitems.alloc(n + 1);
    bcur.zero();
    pitems.zero();
    k_class_count<<<c->sm_count * 4, 256, 0, s>>>(cl.cdeg.p, n, bcur.p);
    k_class_scan<<<1, 32, 0, s>>>(bcur.p);
    k_class_place<<<c->sm_count * 4, 256, 0, s>>>(cl.cdeg.p, items.p, n, bcur.p, perm.p, pitems.p);
    count_launch(3);
  }
  DBuf<uint64_t> item_off(c, s, n + 1), big_off(c, s, n + 1);
  scan_u32(t.peel_order ? pitems.p : items.p, item_off.p, n, c, s);
  scan_u32(multi.p, big_off.p, n, c, s);
  // sized by bounds known on the host, so nothing waits for the scans: a
  // vertex has at most clique degree / item size + 1 items, and a hub more
  // than `chunk` incidences
  const uint64_t nitems = (uint64_t)n + (m * k) / std::min(chunk, hub_chunk) + 1;
  const uint64_t nbig = std::min<uint64_t>(n, (m * k) / chunk + 1);
  if (nitems >= 0xFFFFFFFFull) fail(CDS_ERR_OVERFLOW, "peel: more than 2^32-1 work items");
  DBuf<uint32_t> item_v(c, s, nitems + 1), item_c(c, s, nitems + 1), big_slot(c, s, n),
      big_v(c, s, nbig + 1);
  k_item_fill<<<c->sm_count * 8, 256, 0, s>>>(t.peel_order ? perm.p : nullptr, bcur.p, item_off.p,
                                              big_off.p, n, item_v.p, item_c.p, big_slot.p, big_v.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  DBuf<uint32_t> acc(c, s, nbig * ACC_WORDS + 1), big_done(c, s, nbig + 1);
  acc.zero();
  big_done.zero();
  CDS_CUDA(cudaMemcpyAsync(out.core.p, cl.cdeg.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  DBuf<uint32_t> ctl(c, s, 3 * 32 + 1), ichg(c, s, 3 * (size_t)ninst);
  ichg.zero();
  DBuf<GridBarrier> bar(c, s, 1);
  DBuf<uint32_t> err(c, s, 1);
  ctl.zero();
  bar.zero();
  err.zero();

  HParams p{};
  p.n = n;
  p.k = k;
  p.members = cl.members.p;
  p.inc_off = inc_off.p;
  p.inc = inc.p;
  p.inc64 = inc64.p;
  p.tup = tup.p;
  p.tup16 = tup16.p;
  p.tup64 = tup64.p;
  p.tup_stride = m * k;
  p.tau = out.core.p;
  p.item_v = item_v.p;
  p.item_c = item_c.p;
  p.vitems = items.p;
  p.nitems = item_off.p + n;
  p.chunk = chunk;
  p.hub_chunk = hub_chunk;
  p.big_slot = big_slot.p;
  p.big_v = big_v.p;
  p.nbig = (uint32_t)nbig;
  p.acc = acc.p;
  p.big_done = big_done.p;
  p.ctl = ctl.p;
  p.of_vertex = of_vertex;
  p.ninst = ninst;
  p.ichg = ichg.p;
  p.bar = bar.p;
  p.err = err.p;
  p.spin_limit = 1ull << 26;
  p.max_sweeps = 1u << 20;
  p.time_budget_ns = 120ull * 1000000000ull;
  p.sweeps = ctl.p + 3 * 32;
  DBuf<unsigned long long> reads(c, s, c->prof ? MAX_READ_SWEEPS : 0);
  if (c->prof) reads.zero();
  p.reads = c->prof ? reads.p : nullptr;
  // the static share of the items (peel_static percent, 100: all static)
  p.static_pct = (uint32_t)std::min(100, std::max(0, t.peel_static));
  if (m) {
    void *kern = tuple && narrow ? (k == 2 ? (void *)k_hindex<2, 2>
                                  : k == 3 ? (void *)k_hindex<3, 2> : (void *)k_hindex<4, 2>)
               : tuple && packed ? (k == 3 ? (void *)k_hindex<3, 3> : (void *)k_hindex<4, 3>)
               : tuple ? (k == 2 ? (void *)k_hindex<2, 1>
                        : k == 3 ? (void *)k_hindex<3, 1> : (void *)k_hindex<4, 1>)
               : wide_ids ? (k == 2 ? (void *)k_hindex<2, 4>
                           : k == 3 ? (void *)k_hindex<3, 4>
                           : k == 4 ? (void *)k_hindex<4, 4> : (void *)k_hindex<0, 4>)
                       : (k == 2 ? (void *)k_hindex<2, 0>
                        : k == 3 ? (void *)k_hindex<3, 0>
                        : k == 4 ? (void *)k_hindex<4, 0> : (void *)k_hindex<0, 0>);
    const int threads = 512;
    // each warp's histogram as large as its items need (the rest of the
    // SM's shared memory stays L1, which holds the gathered core values)
    p.warp_words = (std::max<uint32_t>(chunk + 1, ACC_WORDS) + 3u) & ~3u;
    const size_t smem = (size_t)(threads / 32) * p.warp_words * 4;
    CDS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    if (per_sm < 1) fail(CDS_ERR_CUDA, "peel kernel does not fit on an SM");
    per_sm = std::min(per_sm, 2);
    dim3 grid(coop_grid(c, per_sm)), block(threads);
    void *args[] = {&p};
    {
      ProfScope ps(c, s, "peel");
      CDS_CUDA(cudaLaunchCooperativeKernel(kern, grid, block, args, smem, s));
    }
    count_launch();
    CDS_CUDA(cudaGetLastError());
  }
  // the incidence streams are done with (stream-ordered frees), which makes
  // room for the per-clique smallest member core
  tup.release();
  tup16.release();
  tup64.release();
  inc.release();
  inc64.release();
  out.cmin.c = c;
  out.cmin.s = s;
  out.cmin.alloc(m + 1);
  // per-instance largest core (sizes the histograms), read with the status
  DBuf<uint32_t> imax(c, s, ninst);
  imax.zero();
  k_inst_maxcore<<<c->sm_count * 4, 256, 0, s>>>(out.core.p, n, of_vertex, imax.p);
  count_launch();
  uint32_t e = 0;
  {
    HostReads r(s);
    r.add(out.inst_max_core.data(), imax.p, ninst);
    r.add(&e, err.p);
    r.wait();
  }
  if (e & DEV_ERR_TIMEOUT) fail(CDS_ERR_TIMEOUT, "peel: device iteration budget exhausted");
  if (e) fail(CDS_ERR_CUDA, "peel: device error");
  std::vector<uint64_t> hoff(ninst + 1, 0);
  for (uint32_t i = 0; i < ninst; i++) {
    hoff[i + 1] = hoff[i] + out.inst_max_core[i] + 1;
    out.max_core = std::max(out.max_core, out.inst_max_core[i]);
  }
  DBuf<uint64_t> d_hoff(c, s, ninst + 1);
  DBuf<unsigned long long> hv(c, s, hoff[ninst]), hc(c, s, hoff[ninst]);
  DBuf<unsigned long long> bnum(c, s, ninst), bden(c, s, ninst);
  DBuf<uint32_t> ilev(c, s, ninst), blev(c, s, ninst);
  CDS_CUDA(cudaMemcpyAsync(d_hoff.p, hoff.data(), (ninst + 1) * 8, cudaMemcpyHostToDevice, s));
  hv.zero();
  hc.zero();
  {
    ProfScope ps(c, s, "peel_levels");
    k_core_hist<<<c->sm_count * 4, 256, 0, s>>>(out.core.p, n, of_vertex, d_hoff.p, hv.p);
    if (m)
      k_clique_hist<<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, out.core.p, of_vertex,
                                                    d_hoff.p, hc.p, out.cmin.p);
    k_best_level<<<std::min<uint32_t>(ninst, c->sm_count * 4), 512, 0, s>>>(
        d_hoff.p, hv.p, hc.p, ninst, bnum.p, bden.p, ilev.p, blev.p);
    count_launch(m ? 3 : 2);
  }
  CDS_CUDA(cudaGetLastError());
  std::vector<unsigned long long> hn(ninst), hd(ninst);
  uint32_t sweeps = 0;
  {
    HostReads r(s);
    r.add(hn.data(), bnum.p, ninst);
    r.add(hd.data(), bden.p, ninst);
    r.add(out.inst_levels.data(), ilev.p, ninst);
    r.add(out.best_level.data(), blev.p, ninst);
    r.add(&sweeps, p.sweeps);
    r.wait();
  }
  if (c->prof) {
    std::vector<unsigned long long> hr(MAX_READ_SWEEPS);
    {
      HostReads r(s);
      r.add(hr.data(), reads.p, MAX_READ_SWEEPS);
      r.wait();
    }
    std::lock_guard<std::mutex> g(c->mu);
    auto &slot = c->prof_done["peel_sweeps"];
    slot.first += 1;
    slot.second += sweeps;
    // incidences each sweep read, in millions (the early exits skip the rest)
    for (uint32_t i = 0; i < std::min(sweeps, MAX_READ_SWEEPS); i++) {
      char name[32];
      std::snprintf(name, sizeof(name), "peel_reads_sweep%02u", i);
      auto &r2 = c->prof_done[name];
      r2.first += 1;
      r2.second += hr[i] / 1e6;
    }
  }
  for (uint32_t i = 0; i < ninst; i++) {
    out.best_num[i] = hn[i];
    out.best_den[i] = hd[i];
    out.levels = std::max(out.levels, out.inst_levels[i]);
  }
}

}  // namespace cds
