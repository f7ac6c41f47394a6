// flow.cu -- exact densest-subgraph search on the clique-vertex flow network.
//
// Replaces dynamicExactAlgo (cudaCode/main.cu:519-863) with its kernels
// createFlowNetworkOffset / createFlowNetwork / preFlow / pushRelabel /
// globalRelabel / updateFlownetwork (cudaCode/src/helpers.cu:1173-1539), and
// the serial exact() / createFlownetwork / edmondsKarp
// (cpuCode/c++/src/helpers.cpp:1256-1420).
//
// Network (the reference's, cpuCode/c++/src/helpers.cpp:1302-1341), for a
// density guess alpha = p/q with every capacity multiplied by q:
//     s -> v     q * deg(v)        v -> t     k * p
//     v -> psi   q                 psi -> v   q * (k-1)
// The antiparallel pair v <-> psi is one x (flow v -> psi minus flow
// psi -> v; 32-bit when every excursion fits, else 64-bit); residuals are
// q - x and q(k-1) + x.  Max flow = q k |Psi| exactly when no vertex set is
// denser than alpha, and otherwise the vertices that cannot reach t in the
// residual graph form the maximal set maximising |Psi(S)| - alpha |S|, which
// is denser than alpha.
//
// All component networks of a problem (and of every instance of a batch)
// are solved in one cooperative launch of a persistent push-relabel kernel
// at vertex level (clique nodes hold no excess and no label: a push moves
// flow v -> psi -> w in one step):
//   global relabel  BFS from the sinks over residual arcs, level by level
//                   (exact vertex distances; unreachable vertices get INF);
//   rounds          prepare (apply relabels, push to t from label 1, offer
//                   the excess), push (labels frozen: each vertex with an
//                   offer pushes to vertices exactly one lower, a warp per
//                   chunk of its incidence list), relabel (vertices left with
//                   an offer take 1 + the lowest residual neighbour).
// The loop ends when a global relabel finds no active vertex below INF: a
// maximum preflow, whose sink excess is the max-flow value.  Every wait is a
// bounded grid barrier.
#include "device_util.cuh"
#include "stages.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace {

struct FlowParams {
  uint32_t nv;
  uint64_t nc;
  uint32_t k;
  uint32_t *rec;              // [nc << rs] clique records: S member slots (local
                              // vertex ids), then S 32-bit flow words
  uint32_t S, rs;             // slots per record (a power of two >= k), log2(2S)
  const uint64_t *vinc_off;   // [nv+1]
  const void *vinc;           // the cliques of each vertex (record indices), u32 or u64
  const uint32_t *vcnet;      // [nv] network of each vertex
  const uint32_t *chunk_v;    // [nchunks] vertex of each chunk of an incidence list
  const uint64_t *chunk_beg;  // [nchunks] first position of the chunk in vinc
  const uint64_t *nchunks;    // chunks in all, on the device
  uint32_t chunk;
  void *x64;                  // [nc*k] the flow words as int64, when 32 bits do not fit
                              // (flow v -> psi minus flow psi -> v)
  long long *ev, *rt;         // [nv] excess, residual to t
  long long *budget;          // [nv] excess offered to pushes in this round
  int *d, *dnew;              // [nv] labels, relabel targets
  uint8_t *sel;               // [nv] vertex pushes in this round
  long long *sink;            // [nnet]
  const long long *P, *Q;     // alpha per network
  const uint8_t *active;      // [nnet]
  uint32_t *ctl;
  GridBarrier *bar;
  uint32_t *err;
  unsigned long long spin_limit;
  uint32_t max_cycles;
  uint32_t rounds;
  int early_stop;             // -1: exact
  int INF;
  unsigned long long time_budget_ns;  // wall-clock budget of the whole kernel
  unsigned long long *phase_ns;       // [5] block 0's time per phase kind, summed (profiling)
  uint32_t ev_smem;           // pushes add excess in shared memory (nv <= EV_SMEM_MAX)
  unsigned long long *bfs;    // [4] global relabel: incidences of unlabelled vertices,
                              // and of each level's vertices (three slots, by level)
};

// Networks of at most this many vertices, with at least 8 incidences per
// vertex and block of the grid, sum the excess their pushes move in shared
// memory, one copy per block, and add it to ev once per push phase: with
// few vertices and many cliques every push would otherwise be an atomic on
// one of a few hundred words, while with many vertices the flush (up to one
// atomic per vertex and block) costs more than it saves.
constexpr uint32_t EV_SMEM_MAX = 1024;

enum { F_ANY = 0, F_ACTIVE = 3, F_STOPPED = 6, F_CYCLES = 7, F_BFS = 8, F_SEL = 9, F_ROUNDS = 12,
       F_WORDS = 16 };

__device__ __forceinline__ uint64_t chunk_end(const FlowParams &p, uint32_t v, uint64_t b) {
  const uint64_t e = b + p.chunk, ve = p.vinc_off[v + 1];
  return e < ve ? e : ve;
}

// x as 32-bit when every excursion fits (|x| < 2 q k^2 < 2^31), else 64-bit
__device__ __forceinline__ long long atom_add_x(int *a, long long v) {
  return (long long)atomicAdd(a, (int)v);
}
__device__ __forceinline__ long long atom_add_x(long long *a, long long v) {
  return atomic_add_i64(a, v);
}

// The slot of vertex v in a clique's member slots.  An incidence list holds
// only record indices (4 bytes while there are fewer than 2^32 cliques); the
// slot is found among the members, which sit in the same sector as the flow
// words the caller reads next.
__device__ __forceinline__ uint32_t slot_of(const uint32_t *M, uint32_t v, uint32_t k) {
  uint32_t jt = 0;
  for (uint32_t j = 1; j < k; j++) jt = M[j] == v ? j : jt;
  return jt;
}

// A clique's record: its S member slots and its flow words, which share one
// 32-byte sector for k <= 4 (a push reads both for every incidence it
// tries), or its slots in the 64-bit flow array.
__device__ __forceinline__ uint32_t *rec_members(const FlowParams &p, uint64_t c) { return p.rec + (c << p.rs); }
template <typename X>
__device__ __forceinline__ X *rec_flow(const FlowParams &p, uint64_t c) {
  if constexpr (sizeof(X) == 4) return reinterpret_cast<X *>(p.rec + (c << p.rs) + p.S);
  else return reinterpret_cast<X *>(p.x64) + c * p.k;
}

constexpr int FU = 2;  // incidences per lane handled together in push
constexpr int FR = 4;  // and in relabel (no claims there: more loads in flight)

// Atomically takes up to `want` from *b (never below zero) and returns it.
__device__ __forceinline__ long long claim(long long *b, long long want) {
  const long long old = atomic_add_i64(b, -want);
  const long long got = old <= 0 ? 0 : (old < want ? old : want);
  if (got < want) atomic_add_i64(b, want - got);
  return got;
}

// Vertex-level push-relabel.  Clique nodes hold no excess and carry no label:
// a push moves flow v -> psi -> w in one step, admissible when
// d(w) = d(v) - 1 with residual on both arcs, and labels live on vertices
// only, so a global relabel is a BFS over at most n_c vertex levels.
template <typename X, typename I>
__global__ void __launch_bounds__(512, 2) k_flow(FlowParams p) {
  extern __shared__ unsigned long long s_ev[];  // [nv] when p.ev_smem
  const I *const vinc = reinterpret_cast<const I *>(p.vinc);
  volatile uint32_t *ctl = p.ctl;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  const int INF = p.INF;
  const uint32_t k = p.k;
  const uint32_t nchunks = (uint32_t)*p.nchunks;
  // Phase number, +1 per barrier.  Flag slot ph%3 is written in phase ph and
  // read in phase ph+1; the leader clears slot (ph+1)%3 at the start of phase
  // ph, i.e. two phases after its last read and just before its next write.
  uint32_t ph = 0;
  long long last_sink = -1;
  int stale = 0;
  bool done = false;
  // past the budget the leader flags an error that every block sees at the
  // next barrier, so all leave together
  const unsigned long long t0 = globaltimer_ns();
#define BARRIER()                                            \
  do {                                                       \
    if (!grid_sync(p.bar, p.err, p.spin_limit)) return;      \
    ph++;                                                    \
  } while (0)
#define CLEAR_AHEAD()                                                   \
  do {                                                                  \
    if (leader) {                                                       \
      ctl[F_ANY + (ph + 1) % 3] = 0;                                    \
      ctl[F_ACTIVE + (ph + 1) % 3] = 0;                                 \
      ctl[F_SEL + (ph + 1) % 3] = 0;                                    \
      if (globaltimer_ns() - t0 > p.time_budget_ns) atomicOr(p.err, DEV_ERR_TIMEOUT); \
    }                                                                   \
  } while (0)

  // profiling: block 0's time in BFS, activity check, prepare, push, relabel
  unsigned long long tacc[5] = {0, 0, 0, 0, 0}, tprev = globaltimer_ns();
#define PHASE_END(i)                                        \
  do {                                                      \
    if (p.phase_ns && blockIdx.x == 0 && threadIdx.x == 0) { \
      const unsigned long long now = globaltimer_ns();      \
      tacc[i] += now - tprev;                               \
      tprev = now;                                          \
    }                                                       \
  } while (0)
  for (uint32_t cycle = 0; cycle < p.max_cycles; cycle++) {
    // ---------- global relabel: exact vertex distances to t ----------
    // Level-synchronous BFS from the sinks.  Each level either pushes from
    // its vertices (scanning their incidences for unlabelled neighbours) or,
    // when the vertices still unlabelled hold fewer incidences than this
    // level's, pulls: every unlabelled vertex looks for one neighbour at
    // this level and stops at the first.  Both give exact distances.
    CLEAR_AHEAD();
    {
      unsigned long long inf_i = 0, l1_i = 0;
      for (uint32_t v = gtid; v < p.nv; v += gthreads) {
        const bool act = p.active[p.vcnet[v]];
        const bool one = act && p.rt[v] > 0;
        p.d[v] = one ? 1 : INF;
        p.sel[v] = 0;
        p.budget[v] = 0;
        if (act) {
          const unsigned long long inc = p.vinc_off[v + 1] - p.vinc_off[v];
          if (one) l1_i += inc;
          else inf_i += inc;
        }
      }
      inf_i = warp_sum(inf_i);
      l1_i = warp_sum(l1_i);
      if (lane == 0 && inf_i) atomicAdd(&p.bfs[0], inf_i);
      if (lane == 0 && l1_i) atomicAdd(&p.bfs[1 + 1 % 3], l1_i);
    }
    BARRIER();
    unsigned long long inf_rem = *(volatile unsigned long long *)&p.bfs[0];
    for (int lvl = 1; lvl < INF - 1; lvl++) {
      // every block reads the same two words here (nothing writes them in
      // this level), so every block takes the same branch
      const unsigned long long front = *(volatile unsigned long long *)&p.bfs[1 + lvl % 3];
      if (lvl > 1) inf_rem -= front;  // the vertices labelled lvl were unlabelled
      if (inf_rem == 0) break;        // nothing left to reach
      CLEAR_AHEAD();
      // slot (lvl+2)%3 held level lvl-1, read by every block before the
      // barrier that ended that level; it collects level lvl+2
      if (leader) p.bfs[1 + (lvl + 2) % 3] = 0;
      unsigned long long *nextf = p.bfs + 1 + (lvl + 1) % 3;
      bool any = false;
      if (inf_rem >= front) {
        for (uint32_t ch = gwarp; ch < nchunks; ch += nwarps) {
          const uint32_t v = p.chunk_v[ch];
          if (p.d[v] != lvl) continue;
          const long long q = p.Q[p.vcnet[v]];
          const long long qk1 = q * (long long)(k - 1);
          const uint64_t e = chunk_end(p, v, p.chunk_beg[ch]);
          for (uint64_t i = p.chunk_beg[ch] + lane; i < e; i += 32) {
            const uint64_t t = vinc[i];
            const uint64_t cq = t;
            const uint32_t *M = rec_members(p, cq);
            const uint32_t jt = slot_of(M, v, k);
            const X *F = rec_flow<X>(p, cq);
            if (qk1 + F[jt] <= 0) continue;  // no residual psi -> v
            for (uint32_t j = 0; j < k; j++) {
              if (j == jt) continue;
              const uint32_t w = M[j];
              if (q - F[j] > 0 && p.d[w] == INF && atomicCAS(&p.d[w], INF, lvl + 1) == INF) {
                atomicAdd(nextf, (unsigned long long)(p.vinc_off[w + 1] - p.vinc_off[w]));
                any = true;
              }
            }
          }
        }
      } else {
        for (uint32_t ch = gwarp; ch < nchunks; ch += nwarps) {
          const uint32_t w = p.chunk_v[ch];
          if (p.d[w] != INF || !p.active[p.vcnet[w]]) continue;
          const long long q = p.Q[p.vcnet[w]];
          const long long qk1 = q * (long long)(k - 1);
          const uint64_t e = chunk_end(p, w, p.chunk_beg[ch]);
          bool found = false;
          for (uint64_t i0 = p.chunk_beg[ch]; i0 < e && !found; i0 += 32) {
            const uint64_t i = i0 + lane;
            bool f = false;
            if (i < e) {
              const uint64_t tw = vinc[i];
              const uint64_t cq = tw;
              const uint32_t *M = rec_members(p, cq);
              const uint32_t jw = slot_of(M, w, k);
              const X *F = rec_flow<X>(p, cq);
              if (q - F[jw] > 0) {  // residual w -> psi
                for (uint32_t j = 0; j < k && !f; j++) {
                  if (j == jw) continue;
                  f = p.d[M[j]] == lvl && qk1 + F[j] > 0;  // residual psi -> v
                }
              }
            }
            found = __any_sync(CDS_FULL, f);
          }
          if (found && lane == 0 && atomicCAS(&p.d[w], INF, lvl + 1) == INF) {
            atomicAdd(nextf, (unsigned long long)(p.vinc_off[w + 1] - p.vinc_off[w]));
            any = true;
          }
        }
      }
      if (__syncthreads_or(any) && threadIdx.x == 0) ctl[F_ANY + ph % 3] = 1;
      if (leader) ctl[F_BFS] = ctl[F_BFS] + 1;
      const uint32_t slot = ph % 3;
      BARRIER();
      if (!ctl[F_ANY + slot]) break;
    }
    PHASE_END(0);
    // ---------- any active vertex left? ----------
    CLEAR_AHEAD();
    {
      bool act = false;
      for (uint32_t v = gtid; v < p.nv; v += gthreads) act |= p.ev[v] > 0 && p.d[v] < INF;
      if (__syncthreads_or(act) && threadIdx.x == 0) ctl[F_ACTIVE + ph % 3] = 1;
    }
    const uint32_t aslot = ph % 3;
    BARRIER();
    if (!ctl[F_ACTIVE + aslot]) {
      done = true;
      break;
    }
    if (p.early_stop >= 0) {  // opt-in: stop when the sinks stop gaining
      long long tot = 0;      // sink[] is only written in PREPARE phases
      for (uint32_t i = 0; i < p.ctl[F_WORDS]; i++) tot += p.sink[i];
      if (tot == last_sink) stale++;
      else stale = 0;
      last_sink = tot;
      if (stale > p.early_stop) {
        if (leader) ctl[F_STOPPED] = 1;
        break;
      }
    }
    PHASE_END(1);
    // ---------- rounds: prepare, push, relabel ----------
    for (uint32_t r = 0; r < p.rounds; r++) {
      // PREPARE (thread per vertex): apply last round's relabels, push to t
      // from label 1, and offer the remaining excess to this round
      CLEAR_AHEAD();
      // the global relabel's counters are read by no block any more (every
      // block passed the barrier after the activity check): clear them for
      // the next cycle
      if (leader && r == 0)
        for (int i = 0; i < 4; i++) p.bfs[i] = 0;
      bool any_sel = false;
      for (uint32_t v = gtid; v < p.nv; v += gthreads) {
        if (p.sel[v] && p.budget[v] > 0) p.d[v] = p.dnew[v];
        p.dnew[v] = INF;
        const uint32_t net = p.vcnet[v];
        long long e = p.ev[v];
        if (!p.active[net] || e <= 0 || p.d[v] >= INF) {
          p.sel[v] = 0;
          p.budget[v] = 0;
          continue;
        }
        if (p.d[v] == 1 && p.rt[v] > 0) {
          const long long dl = e < p.rt[v] ? e : p.rt[v];
          p.rt[v] -= dl;
          p.ev[v] = e - dl;
          e -= dl;
          atomic_add_i64(&p.sink[net], dl);
        }
        p.budget[v] = e;
        p.sel[v] = e > 0;
        any_sel |= e > 0;
      }
      if (__syncthreads_or(any_sel) && threadIdx.x == 0) ctl[F_SEL + ph % 3] = 1;
      if (leader) ctl[F_ROUNDS] = ctl[F_ROUNDS] + 1;
      const uint32_t sslot = ph % 3;
      BARRIER();
      PHASE_END(2);
      // nothing to push below INF: the next global relabel decides
      if (!ctl[F_SEL + sslot]) break;
      // PUSH (warp per chunk): v -> psi -> w with d(w) = d(v) - 1
      CLEAR_AHEAD();
      if (p.ev_smem) {
        for (uint32_t i = threadIdx.x; i < p.nv; i += blockDim.x) s_ev[i] = 0;
        __syncthreads();
      }
      for (uint32_t ch = gwarp; ch < nchunks; ch += nwarps) {
        const uint32_t v = p.chunk_v[ch];
        if (!p.sel[v]) continue;
        const int dv = p.d[v];
        if (dv <= 1) continue;
        const long long q = p.Q[p.vcnet[v]];
        const long long qk1 = q * (long long)(k - 1);
        const uint64_t e = chunk_end(p, v, p.chunk_beg[ch]);
        long long pushed_w = 0;
        // FU incidences per lane at a time: their capacities first (every
        // load in flight together), one claim on v's budget for all of
        // them, then the pushes.  The budget is read once per chunk; after
        // that a claim that got less than it asked for shows it is spent.
        {
          long long left = 0;
          if (lane == 0) left = *(volatile long long *)&p.budget[v];
          if (__shfl_sync(CDS_FULL, left, 0) <= 0) continue;
        }
        // the next step's incidence ids load while this step runs
        I tn[FU];
#pragma unroll
        for (int u = 0; u < FU; u++) {
          const uint64_t i = p.chunk_beg[ch] + 32u * u + lane;
          tn[u] = i < e ? vinc[i] : (I)0;
        }
        for (uint64_t i0 = p.chunk_beg[ch]; i0 < e; i0 += 32 * FU) {
          uint64_t t[FU];
          long long cap[FU];
#pragma unroll
          for (int u = 0; u < FU; u++) t[u] = i0 + 32u * u + lane < e ? (uint64_t)tn[u] : ~0ull;
#pragma unroll
          for (int u = 0; u < FU; u++) {
            const uint64_t i = i0 + 32u * (FU + u) + lane;
            tn[u] = i < e ? vinc[i] : (I)0;
          }
#pragma unroll
          for (int u = 0; u < FU; u++) {
            cap[u] = 0;
            if (t[u] == ~0ull) continue;
            const uint64_t cq = t[u];
            const uint32_t *M = rec_members(p, cq);
            const uint32_t jt = slot_of(M, v, k);
            const X *F = rec_flow<X>(p, cq);
            const long long r1 = q - F[jt];
            if (r1 <= 0) continue;
            long long s2 = 0;
            for (uint32_t j = 0; j < k; j++) {
              if (j == jt || p.d[M[j]] != dv - 1) continue;
              const long long r2 = qk1 + F[j];
              if (r2 > 0) s2 += r2;
            }
            cap[u] = r1 < s2 ? r1 : s2;
          }
          // this lane's capacities in order, then the lanes in order
          long long mine = 0;
#pragma unroll
          for (int u = 0; u < FU; u++) mine += cap[u];
          const long long incl = warp_inclusive_scan(mine);
          const long long tot = __shfl_sync(CDS_FULL, incl, 31);
          if (tot == 0) continue;
          long long got = 0;
          if (lane == 0) got = claim(&p.budget[v], tot);
          got = __shfl_sync(CDS_FULL, got, 0);
          long long before = incl - mine;  // capacity of the lanes before this one
          long long unused_l = 0, act_l = 0;
#pragma unroll
          for (int u = 0; u < FU; u++) {
            long long share = got - before;
            share = share < 0 ? 0 : (share > cap[u] ? cap[u] : share);
            before += cap[u];
            if (share <= 0) continue;
            const uint64_t cq = t[u];
            const uint32_t *M = rec_members(p, cq);
            const uint32_t jt = slot_of(M, v, k);
            X *F = rec_flow<X>(p, cq);
            long long act = 0;
            for (uint32_t j = 0; j < k && act < share; j++) {
              if (j == jt) continue;
              const uint32_t w = M[j];
              if (p.d[w] != dv - 1) continue;
              const long long r2 = qk1 + F[j];
              if (r2 <= 0) continue;
              const long long want = (share - act) < r2 ? (share - act) : r2;
              // reserve on psi -> w; give back what another sender took first
              const long long old = atom_add_x(&F[j], -want);
              const long long avail = qk1 + old;
              const long long ok = avail <= 0 ? 0 : (avail < want ? avail : want);
              if (ok < want) atom_add_x(&F[j], want - ok);
              if (ok > 0) {
                if (p.ev_smem) atomicAdd(&s_ev[w], (unsigned long long)ok);
                else atomic_add_i64(&p.ev[w], ok);
                act += ok;
              }
            }
            if (act > 0) atom_add_x(&F[jt], act);
            act_l += act;
            unused_l += share - act;
          }
          const long long unused = warp_sum(unused_l);
          pushed_w += warp_sum(act_l);
          if (lane == 0 && unused > 0) atomic_add_i64(&p.budget[v], unused);
          if (got < tot) break;  // the budget ran out with this claim
        }
        if (lane == 0 && pushed_w > 0) {
          if (p.ev_smem) atomicAdd(&s_ev[v], (unsigned long long)(-pushed_w));
          else atomic_add_i64(&p.ev[v], -pushed_w);
        }
      }
      if (p.ev_smem) {  // this block's net excess changes, once per vertex
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < p.nv; i += blockDim.x)
          if (s_ev[i]) atomic_add_i64(&p.ev[i], (long long)s_ev[i]);
      }
      BARRIER();
      PHASE_END(3);
      // RELABEL (warp per chunk) for vertices that kept part of their offer
      CLEAR_AHEAD();
      for (uint32_t ch = gwarp; ch < nchunks; ch += nwarps) {
        const uint32_t v = p.chunk_v[ch];
        if (!p.sel[v] || p.budget[v] <= 0) continue;
        const long long q = p.Q[p.vcnet[v]];
        const long long qk1 = q * (long long)(k - 1);
        const uint64_t e = chunk_end(p, v, p.chunk_beg[ch]);
        int mn = INF;
        if (lane == 0 && p.chunk_beg[ch] == p.vinc_off[v] && p.rt[v] > 0) mn = 0;
        for (uint64_t i0 = p.chunk_beg[ch] + lane; i0 < e; i0 += 32 * FR) {
          uint64_t t[FR];
#pragma unroll
          for (int u = 0; u < FR; u++) t[u] = i0 + 32u * u < e ? (uint64_t)vinc[i0 + 32u * u] : ~0ull;
#pragma unroll
          for (int u = 0; u < FR; u++) {
            if (t[u] == ~0ull) continue;
            const uint64_t cq = t[u];
            const uint32_t *M = rec_members(p, cq);
            const uint32_t jt = slot_of(M, v, k);
            const X *F = rec_flow<X>(p, cq);
            if (q - F[jt] <= 0) continue;
            for (uint32_t j = 0; j < k; j++) {
              if (j == jt || qk1 + F[j] <= 0) continue;
              const int dw = p.d[M[j]];
              mn = dw < mn ? dw : mn;
            }
          }
        }
        mn = warp_min(mn);
        if (lane == 0) atomicMin(&p.dnew[v], mn >= INF - 1 ? INF : mn + 1);
      }
      BARRIER();
      PHASE_END(4);
    }
    if (leader) ctl[F_CYCLES] = cycle + 1;
  }
  if (p.phase_ns && blockIdx.x == 0 && threadIdx.x == 0)
    for (int i = 0; i < 5; i++) p.phase_ns[i] += tacc[i];
  if (!done && !ctl[F_STOPPED] && leader) atomicOr(p.err, DEV_ERR_TIMEOUT);
#undef PHASE_END
#undef BARRIER
#undef CLEAR_AHEAD
}

// Warm start (before a preflow): a balanced split of every clique's k q
// units among its members.  Any split is a valid flow state (member j keeps
// a_j of the units, x_j = q - a_j lies in [-q(k-1), q] and the x of a clique
// sum to 0), and the closer every member's load is to its sink capacity k p,
// the less excess the push-relabel has to move.  Weights w(v) give the split
// a_j ~ w(v_j); they start at 1 / clique degree and take multiplicative
// updates w(v) *= (k p / q) / load(v) (loads in units of q) -- the
// proportional-response iteration for the fractional densest-subgraph
// assignment.  On the 110-vertex densest core of the R-MAT-14 k = 4 graph
// one split leaves 2.9 % of the units as excess instead of 14 %, two
// updates and the split 0.7 % (the split's CPU restatement in the flow
// model tests gives these figures).
constexpr uint32_t SPLIT_SMEM_NV = 4096;  // per-block load sums in shared memory up to here

__global__ void k_split_init(FlowParams p, float *__restrict__ w) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < p.nv; v += gridDim.x * blockDim.x) {
    const uint64_t d = p.vinc_off[v + 1] - p.vinc_off[v];
    w[v] = d ? 1.0f / (float)d : 1.0f;
  }
}

// loads of the split the weights give, in units of q (K = k for k <= 4,
// so the member arrays stay in registers; 0: any k)
template <int K>
__global__ void k_split_loads(FlowParams p, const float *__restrict__ w, float *__restrict__ load) {
  __shared__ float s_l[SPLIT_SMEM_NV];
  const bool sm = p.nv <= SPLIT_SMEM_NV;
  if (sm) {
    for (uint32_t v = threadIdx.x; v < p.nv; v += blockDim.x) s_l[v] = 0.0f;
    __syncthreads();
  }
  const uint32_t k = K ? K : p.k;
  constexpr int A = K ? K : 16;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < p.nc; b += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = b + threadIdx.x;
    uint32_t mem[A];
    float ws[A], sum = 0.0f;
    bool in = c < p.nc;
    if (in) {
      const uint32_t *M = rec_members(p, c);
#pragma unroll
      for (int j = 0; j < A; j++)
        if (j < (int)k) {
          mem[j] = M[j];
          ws[j] = w[mem[j]];
          sum += ws[j];
        }
      in = p.active[p.vcnet[mem[0]]];
    }
    const float f = in ? (float)k / sum : 0.0f;
    // the last member changes from one clique to the next (it is the
    // innermost of the listing's loops): a plain atomic; the others repeat
    // over runs of lanes, summed first
#pragma unroll
    for (int j = 0; j < A; j++) {
      if (j + 1 < (int)k) run_add(sm ? s_l : load, in ? mem[j] : 0u, in ? ws[j] * f : 0.0f, in);
      else if (j + 1 == (int)k && in) atomicAdd(sm ? &s_l[mem[j]] : &load[mem[j]], ws[j] * f);
    }
  }
  if (sm) {
    __syncthreads();
    for (uint32_t v = threadIdx.x; v < p.nv; v += blockDim.x)
      if (s_l[v] != 0.0f) atomicAdd(&load[v], s_l[v]);
  }
}

__global__ void k_split_update(FlowParams p, float *__restrict__ w, float *__restrict__ load) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < p.nv; v += gridDim.x * blockDim.x) {
    const uint32_t net = p.vcnet[v];
    const float l = load[v];
    load[v] = 0.0f;
    if (!p.active[net] || !(l > 0.0f)) continue;
    const float cap = (float)p.k * (float)((double)p.P[net] / (double)p.Q[net]);
    w[v] = fminf(fmaxf(w[v] * (cap / l), 1e-30f), 1e30f);
  }
}

// The split as flow state, in exact integers: a_j = floor(k q w_j / sum) for
// every slot but the one of largest weight, which takes the rest, so the a_j
// sum to k q and each lies in [0, k q]; `units` collects each vertex's a_j.
template <typename X, int K>
__global__ void k_split_apply(FlowParams p, const float *__restrict__ w, unsigned long long *__restrict__ units) {
  __shared__ unsigned long long s_u[SPLIT_SMEM_NV];
  const bool sm = p.nv <= SPLIT_SMEM_NV;
  if (sm) {
    for (uint32_t v = threadIdx.x; v < p.nv; v += blockDim.x) s_u[v] = 0;
    __syncthreads();
  }
  const uint32_t k = K ? K : p.k;
  constexpr int A = K ? K : 16;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < p.nc; b += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = b + threadIdx.x;
    uint32_t mem[A];
    unsigned long long a[A];
    bool in = c < p.nc;
    if (in) {
      const uint32_t *M = rec_members(p, c);
      float ws[A];
      float sum = 0.0f, wmax = -1.0f;
      uint32_t jm = 0;
#pragma unroll
      for (int j = 0; j < A; j++)
        if (j < (int)k) {
          mem[j] = M[j];
          ws[j] = w[mem[j]];
          sum += ws[j];
          if (ws[j] > wmax) {
            wmax = ws[j];
            jm = j;
          }
        }
      const uint32_t net = p.vcnet[mem[0]];
      in = p.active[net];
      if (in) {
        X *F = rec_flow<X>(p, c);
        const long long q = p.Q[net], kq = (long long)k * q;
        long long acc = 0;
#pragma unroll
        for (int j = 0; j < A; j++)
          if (j < (int)k && j != (int)jm) {
            long long x = (long long)((double)kq * (double)(ws[j] / sum));
            x = x < 0 ? 0 : (x > kq - acc ? kq - acc : x);
            acc += x;
            a[j] = (unsigned long long)x;
          }
#pragma unroll
        for (int j = 0; j < A; j++)
          if (j == (int)jm) a[j] = (unsigned long long)(kq - acc);
#pragma unroll
        for (int j = 0; j < A; j++)
          if (j < (int)k) F[j] = (X)(q - (long long)a[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < A; j++) {
      if (j + 1 < (int)k) run_add(sm ? s_u : units, in ? mem[j] : 0u, in ? a[j] : 0ull, in);
      else if (j + 1 == (int)k && in && a[j]) atomicAdd(sm ? &s_u[mem[j]] : &units[mem[j]], a[j]);
    }
  }
  if (sm) {
    __syncthreads();
    for (uint32_t v = threadIdx.x; v < p.nv; v += blockDim.x)
      if (s_u[v]) atomicAdd(&units[v], s_u[v]);
  }
}

// preflow: saturate s -> v, then v -> t as far as it goes.  With a warm start
// v's excess is the units it holds (s supplies q per clique, and v passed
// q - x of each into the clique); without one, x = 0 and it is q deg(v).
__global__ void k_preflow(FlowParams p, const unsigned long long *__restrict__ load) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < p.nv; v += gridDim.x * blockDim.x) {
    const uint32_t net = p.vcnet[v];
    if (!p.active[net]) continue;
    const long long q = p.Q[net], kp = (long long)p.k * p.P[net];
    const long long supply = load ? (long long)load[v] : q * (long long)(p.vinc_off[v + 1] - p.vinc_off[v]);
    const long long f = supply < kp ? supply : kp;
    p.ev[v] = supply - f;
    p.rt[v] = kp - f;
    if (f) atomic_add_i64(&p.sink[net], f);
  }
}

template <typename X>
__global__ void k_reset_flow(FlowParams p) {
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < p.nc;
       c += (uint64_t)gridDim.x * blockDim.x) {
    if (!p.active[p.vcnet[rec_members(p, c)[0]]]) continue;
    X *F = rec_flow<X>(p, c);
    for (uint32_t j = 0; j < p.k; j++) F[j] = 0;
  }
}

// size and clique count of the unreachable side of every active network
// (vertices and cliques are grouped by network: one atomic per warp mostly)
__global__ void k_cut_stats(FlowParams p, unsigned long long *sz, unsigned long long *cnt) {
  const uint32_t stride = gridDim.x * blockDim.x;
  RunCount run;
  for (uint32_t b = blockIdx.x * blockDim.x; b < p.nv; b += stride) {
    const uint32_t v = b + threadIdx.x;
    uint32_t net = 0;
    bool in = false;
    if (v < p.nv) {
      net = p.vcnet[v];
      in = p.active[net] && p.d[v] >= p.INF;
    }
    run.add(sz, net, in);
  }
  run.flush(sz);
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < p.nc; b += stride) {
    const uint64_t c = b + threadIdx.x;
    uint32_t net = 0;
    bool in = false;
    if (c < p.nc) {
      const uint32_t *M = rec_members(p, c);
      net = p.vcnet[M[0]];
      in = p.active[net];
      for (uint32_t j = 0; j < p.k && in; j++) in = p.d[M[j]] >= p.INF;
    }
    run.add(cnt, net, in);
  }
  run.flush(cnt);
}

// remember the unreachable side of the networks that just finished
__global__ void k_mark_answer(const FlowParams p, const uint8_t *fin, uint8_t *mark) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < p.nv; v += gridDim.x * blockDim.x) {
    const uint32_t net = p.vcnet[v];
    if (fin[net]) mark[v] = p.d[v] >= p.INF;
  }
}

// chunks of every incidence list: count, then fill after a scan
__global__ void k_chunk_count(const uint64_t *vinc_off, uint32_t nv, uint32_t chunk, uint32_t *cnt) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    cnt[v] = (uint32_t)((vinc_off[v + 1] - vinc_off[v] + chunk - 1) / chunk);
}
__global__ void k_chunk_fill(const uint64_t *vinc_off, uint32_t nv, uint32_t chunk,
                             const uint64_t *first, uint32_t *chunk_v, uint64_t *chunk_beg) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const uint64_t n = first[v + 1] - first[v];
    for (uint64_t i = 0; i < n; i++) {
      chunk_v[first[v] + i] = v;
      chunk_beg[first[v] + i] = vinc_off[v] + i * chunk;
    }
  }
}

__global__ void k_collect(const uint8_t *mark, const uint32_t *vcnet, const uint32_t *vmap,
                          uint32_t nv, const uint8_t *want, uint32_t *out, uint32_t *cnt) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    if (mark[v] && want[vcnet[v]]) out[atomicAdd(cnt, 1u)] = vmap[v];
}

int64_t gcd64(int64_t a, int64_t b) {
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}
// a/b < c/d, positive denominators
bool frac_lt(int64_t a, int64_t b, int64_t c, int64_t d) {
  return (__int128)a * d < (__int128)c * b;
}

struct CompState {
  bool candidate = false, done = false, improved = false;
  int64_t lb_n = 0, lb_d = 1;  // best density found (lower bound)
  int64_t ub_n = 0, ub_d = 1;  // upper bound (bisection)
  int64_t an = 0, ad = 1;      // current probe
  bool certify = false;        // current probe is at alpha = lb
  bool cut_short = false;      // ended by early stop, not by a certificate
};

}  // namespace

namespace cds {

void exact_search(cds_ctx *c, cudaStream_t s, const CoreOut &co, const Instances &inst,
                  uint32_t k, const cds_params &prm, const Tuning &t, FlowAnswer &ans) {
  const uint32_t ninst = inst.count;
  const uint32_t nnet = co.ncomp;
  ans.num.assign(ninst, 0);
  ans.den.assign(ninst, 0);
  ans.set.assign(ninst, {});
  ans.flows = 0;
  ans.early_stopped = 0;
  ans.ub_num.assign(ninst, 0);
  ans.ub_den.assign(ninst, 1);
  ans.comp_inst.assign(co.comp_inst.begin(), co.comp_inst.end());
  ans.comp_lb.assign(nnet, 0.0);
  ans.comp_ub.assign(nnet, 0.0);
  if (nnet == 0) return;
  const uint32_t nv = co.comp_vbeg[nnet];
  const uint64_t nc = co.comp_cbeg[nnet];

  // starting answer of every instance: its densest whole component (first on ties)
  std::vector<int64_t> best_n(ninst, 0), best_d(ninst, 0);
  std::vector<int32_t> best_comp(ninst, -1);
  std::vector<bool> best_is_whole(ninst, true);
  for (uint32_t i = 0; i < nnet; i++) {
    const uint32_t in = co.comp_inst[i];
    const int64_t cn = (int64_t)(co.comp_cbeg[i + 1] - co.comp_cbeg[i]);
    const int64_t cd = (int64_t)(co.comp_vbeg[i + 1] - co.comp_vbeg[i]);
    if (best_comp[in] < 0 || frac_lt(best_n[in], best_d[in], cn, cd)) {
      best_n[in] = cn;
      best_d[in] = cd;
      best_comp[in] = (int32_t)i;
    }
  }
  std::vector<CompState> st(nnet);
  uint32_t ncand = 0;
  for (uint32_t i = 0; i < nnet; i++) {
    const uint32_t in = co.comp_inst[i];
    const int64_t mc = (int64_t)(co.comp_cbeg[i + 1] - co.comp_cbeg[i]);
    // upper bounds: the largest core number inside, and |Psi_c|^((k-1)/k) / (k!)^(1/k)
    long double lf = 0;
    for (uint32_t j = 2; j <= k; j++) lf += std::log((long double)j);
    const long double ub1 = std::exp(((long double)k - 1) / k * std::log((long double)mc) - lf / k);
    const long double ubf = std::min<long double>((long double)co.comp_maxcore[i], ub1);
    const long double bestf = (long double)best_n[in] / (long double)best_d[in];
    ans.comp_lb[i] = (double)bestf;
    ans.comp_ub[i] = (double)ub1;
    if (ubf * (1 + 1e-12L) + 1e-12L <= bestf) continue;  // cannot beat the starting answer
    CompState &cs = st[i];
    cs.candidate = true;
    cs.lb_n = best_n[in];
    cs.lb_d = best_d[in];
    cs.ub_n = (int64_t)co.comp_maxcore[i];
    cs.ub_d = 1;
    ncand++;
  }

  // flow state width: 32-bit when every probe's q keeps 2 q k^2 < 2^31 (q is
  // a set size with Dinkelbach probes, at most n_c (n_c - 1) with bisection)
  __int128 qbound = 1;
  for (uint32_t i = 0; i < nnet; i++) {
    const __int128 nci = (__int128)(co.comp_vbeg[i + 1] - co.comp_vbeg[i]);
    qbound = std::max<__int128>(qbound, prm.search == 1 ? nci * std::max<__int128>(nci - 1, 1) : nci);
  }
  const bool x32_fits =
      !(c->flags & CDS_CONFIG_WIDE_FLOW) && (__int128)2 * qbound * k * k < ((__int128)1 << 31);
  FlowParams p{};
  // 32-bit flow words live in the clique records; 64-bit ones in their own array
  DBuf<long long> x(c, s, x32_fits ? 0 : nc * k + 1), ev(c, s, nv + 1), rt(c, s, nv + 1),
      budget(c, s, nv + 1);
  DBuf<int> d(c, s, nv + 1), dnew(c, s, nv + 1);
  DBuf<uint8_t> sel(c, s, nv + 1), mark(c, s, nv + 1);
  DBuf<long long> sink(c, s, nnet), P(c, s, nnet), Q(c, s, nnet);
  DBuf<uint8_t> active(c, s, nnet), fin(c, s, nnet);
  DBuf<uint32_t> ctl(c, s, F_WORDS + 1);
  DBuf<GridBarrier> bar(c, s, 1);
  DBuf<uint32_t> err(c, s, 1);
  DBuf<unsigned long long> cut(c, s, 2 * (size_t)nnet);
  DBuf<unsigned long long> bfsw(c, s, 4);
  // warm start: T - 1 weight updates, then the split (t.flow_warm; < 0: by
  // size, three for networks of a million cliques or more; 0: none)
  const uint32_t T = (uint32_t)std::min(255, t.flow_warm < 0 ? (nc >= (1ull << 20) ? 3 : 0) : t.flow_warm);
  DBuf<float> wgt(c, s, T ? nv + 1 : 0), wl(c, s, T ? nv + 1 : 0);
  DBuf<unsigned long long> wload(c, s, T ? nv + 1 : 0);
  bool wgt_init = false;
  sel.zero();
  mark.zero();
  budget.zero();
  const int threads = std::min(512, std::max(128, t.flow_block)) & ~31;  // whole warps
  const uint64_t max_blocks = (uint64_t)c->sm_count * 2;
  const size_t ev_bytes =
      nv <= EV_SMEM_MAX && (uint64_t)nv * max_blocks * 8 <= nc * k ? (size_t)nv * 8 : 0;
  int per_sm = 0;
  {
    int a = 0, b = 0;
    CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_flow<int, uint64_t>, threads, ev_bytes));
    CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_flow<long long, uint64_t>, threads, ev_bytes));
    per_sm = std::min(a, b);
  }
  if (per_sm < 1) fail(CDS_ERR_CUDA, "flow kernel does not fit on an SM");
  per_sm = std::min(per_sm, 2);
  const int G = c->sm_count * 4;
  // the grid: the whole device, or (flow_inc_per_block) one block per that
  // many incidences, at least 8 -- a barrier among fewer blocks is cheaper,
  // which is what the many short phases of a small network wait on
  unsigned blocks = coop_grid(c, per_sm);
  if (t.flow_inc_per_block > 0) {
    const uint64_t want = (nc * k + (uint64_t)t.flow_inc_per_block - 1) / (uint64_t)t.flow_inc_per_block;
    blocks = (unsigned)std::max<uint64_t>(std::min<uint64_t>(8, blocks), std::min<uint64_t>(blocks, want));
  }
  // incidence lists cut into chunks, about four per warp of the grid
  const uint64_t warps = (uint64_t)blocks * threads / 32;
  uint32_t chunk = (uint32_t)std::min<uint64_t>(4096, std::max<uint64_t>(32, (nc * k) / (4 * warps + 1)));
  chunk = (chunk + 31) & ~31u;
  DBuf<uint32_t> nch(c, s, nv + 1);
  DBuf<uint64_t> first(c, s, nv + 1);
  k_chunk_count<<<G, 256, 0, s>>>(co.vinc_off.p, nv, chunk, nch.p);
  count_launch();
  scan_u32(nch.p, first.p, nv, c, s);
  // sized by a bound (ceil(deg / chunk) <= deg / chunk + 1 per vertex), so
  // nothing waits for the scan; the kernels read the count on the device
  const uint64_t nchunks = (nc * k) / chunk + nv + 1;
  if (nchunks >= 0xFFFFFFFFull) fail(CDS_ERR_OVERFLOW, "too many incidence chunks");
  DBuf<uint32_t> chunk_v(c, s, nchunks + 1);
  DBuf<uint64_t> chunk_beg(c, s, nchunks + 1);
  k_chunk_fill<<<G, 256, 0, s>>>(co.vinc_off.p, nv, chunk, first.p, chunk_v.p, chunk_beg.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  p.nv = nv;
  p.nc = nc;
  p.k = k;
  p.rec = co.rec.p;
  p.S = rec_slots(k);
  p.rs = rec_shift(k);
  p.vinc_off = co.vinc_off.p;
  p.vinc = co.vinc.p;
  p.vcnet = co.vcnet.p;
  p.chunk_v = chunk_v.p;
  p.chunk_beg = chunk_beg.p;
  p.nchunks = first.p + nv;
  p.chunk = chunk;
  p.x64 = x.p;
  p.ev = ev.p;
  p.rt = rt.p;
  p.budget = budget.p;
  p.d = d.p;
  p.dnew = dnew.p;
  p.sel = sel.p;
  p.sink = sink.p;
  p.P = P.p;
  p.Q = Q.p;
  p.active = active.p;
  p.ctl = ctl.p;
  p.bar = bar.p;
  p.err = err.p;
  p.spin_limit = 1ull << 24;
  p.max_cycles = 1u << 20;
  p.time_budget_ns = 120ull * 1000000000ull;
  DBuf<unsigned long long> phase(c, s, 5);
  phase.zero();
  p.phase_ns = c->prof ? phase.p : nullptr;
  p.rounds = (uint32_t)std::max(1, t.flow_rounds);
  p.early_stop = prm.early_stop;
  p.INF = (int)std::min<uint64_t>((uint64_t)nv + 2, 1u << 30);
  p.ev_smem = ev_bytes ? 1u : 0u;
  p.bfs = bfsw.p;

  std::vector<long long> hP(nnet), hQ(nnet);
  std::vector<uint8_t> hact(nnet), hfin(nnet);

  bool fresh = co.flows_zero;  // record flow words untouched since they were built
  co.flows_zero = false;
  while (ncand) {
    // choose the probe of every open network
    for (uint32_t i = 0; i < nnet; i++) {
      CompState &cs = st[i];
      hact[i] = 0;
      if (!cs.candidate || cs.done) continue;
      const int64_t nci = (int64_t)(co.comp_vbeg[i + 1] - co.comp_vbeg[i]);
      const int64_t mci = (int64_t)(co.comp_cbeg[i + 1] - co.comp_cbeg[i]);
      cs.an = cs.lb_n;
      cs.ad = cs.lb_d;
      cs.certify = true;
      if (prm.search == 1) {
        // bisection on the grid j / D, D = n_c (n_c - 1), while a grid point
        // lies strictly between the bounds and the scaled capacities fit
        const int64_t D = nci * (nci - 1);
        const bool fits = D > 0 && (__int128)D * k * mci < ((__int128)1 << 62);
        if (fits && frac_lt(cs.lb_n, cs.lb_d, cs.ub_n, cs.ub_d)) {
          // gap >= 1/D ?
          const __int128 gap_num = (__int128)cs.ub_n * cs.lb_d - (__int128)cs.lb_n * cs.ub_d;
          const __int128 gap_den = (__int128)cs.ub_d * cs.lb_d;
          if (gap_num * D >= gap_den) {
            const __int128 mid = ((__int128)cs.lb_n * cs.ub_d + (__int128)cs.ub_n * cs.lb_d) * D /
                                 (2 * (__int128)cs.lb_d * cs.ub_d);
            const int64_t j = (int64_t)mid;
            if (frac_lt(cs.lb_n, cs.lb_d, j, D) && frac_lt(j, D, cs.ub_n, cs.ub_d)) {
              cs.an = j;
              cs.ad = D;
              cs.certify = false;
            }
          }
        }
      }
      const int64_t g = gcd64(cs.an, cs.ad);
      hP[i] = cs.an / g;
      hQ[i] = cs.ad / g;
      if ((__int128)hQ[i] * k * mci >= ((__int128)1 << 62) || (__int128)hP[i] * k >= ((__int128)1 << 62))
        fail(CDS_ERR_OVERFLOW, "flow capacities exceed 62 bits");
      hact[i] = 1;
    }
    CDS_CUDA(cudaMemcpyAsync(P.p, hP.data(), nnet * 8, cudaMemcpyHostToDevice, s));
    CDS_CUDA(cudaMemcpyAsync(Q.p, hQ.data(), nnet * 8, cudaMemcpyHostToDevice, s));
    CDS_CUDA(cudaMemcpyAsync(active.p, hact.data(), nnet, cudaMemcpyHostToDevice, s));
    sink.zero();
    ctl.zero();
    bar.zero();
    err.zero();
    bfsw.zero();
    {
      uint32_t nn = nnet;
      CDS_CUDA(cudaMemcpyAsync(ctl.p + F_WORDS, &nn, 4, cudaMemcpyHostToDevice, s));
    }
    // 32-bit flow state when every excursion of x fits: |x| <= q(k-1) plus
    // at most k-1 concurrent reservations of up to qk each
    long long qmax = 1;
    for (uint32_t i = 0; i < nnet; i++)
      if (hact[i]) qmax = std::max<long long>(qmax, hQ[i]);
    const bool x32 = x32_fits && (__int128)2 * qmax * k * k < ((__int128)1 << 31);
    if (x32_fits && !x32) fail(CDS_ERR_OVERFLOW, "flow probe outside the bound its state was sized for");
    if (!T && !(x32 && fresh)) {  // the split writes every active clique's flows
      if (x32) k_reset_flow<int><<<G, 256, 0, s>>>(p);
      else k_reset_flow<long long><<<G, 256, 0, s>>>(p);
      count_launch();
    }
    fresh = false;
    if (T) {
      ProfScope ps(c, s, "flow_warm");
      if (!wgt_init) {  // the weights carry over between the probes
        wl.zero();
        k_split_init<<<G, 256, 0, s>>>(p, wgt.p);
        count_launch();
        wgt_init = true;
      }
      for (uint32_t r = 1; r < T; r++) {
        if (k == 3) k_split_loads<3><<<G, 256, 0, s>>>(p, wgt.p, wl.p);
        else if (k == 4) k_split_loads<4><<<G, 256, 0, s>>>(p, wgt.p, wl.p);
        else k_split_loads<0><<<G, 256, 0, s>>>(p, wgt.p, wl.p);
        k_split_update<<<G, 256, 0, s>>>(p, wgt.p, wl.p);
        count_launch(2);
      }
      wload.zero();
      if (x32 && k == 3) k_split_apply<int, 3><<<G, 256, 0, s>>>(p, wgt.p, wload.p);
      else if (x32 && k == 4) k_split_apply<int, 4><<<G, 256, 0, s>>>(p, wgt.p, wload.p);
      else if (x32) k_split_apply<int, 0><<<G, 256, 0, s>>>(p, wgt.p, wload.p);
      else k_split_apply<long long, 0><<<G, 256, 0, s>>>(p, wgt.p, wload.p);
      count_launch();
    }
    k_preflow<<<G, 256, 0, s>>>(p, T ? wload.p : nullptr);
    count_launch();
    CDS_CUDA(cudaGetLastError());
    dim3 grid(blocks), block((unsigned)threads);
    void *args[] = {&p};
    {
      ProfScope ps(c, s, "push_relabel");
      void *kern = co.vinc_wide ? (x32 ? (void *)k_flow<int, uint64_t> : (void *)k_flow<long long, uint64_t>)
                                : (x32 ? (void *)k_flow<int, uint32_t> : (void *)k_flow<long long, uint32_t>);
      CDS_CUDA(cudaLaunchCooperativeKernel(kern, grid, block, args, ev_bytes, s));
    }
    count_launch();
    CDS_CUDA(cudaGetLastError());
    cut.zero();
    k_cut_stats<<<G, 256, 0, s>>>(p, cut.p, cut.p + nnet);
    count_launch();
    CDS_CUDA(cudaGetLastError());
    std::vector<long long> hsink(nnet);
    std::vector<unsigned long long> hcut(2 * (size_t)nnet);
    uint32_t hctl[F_WORDS];
    uint32_t herr = 0;
    {
      HostReads r(s);
      r.add(hsink.data(), sink.p, nnet);
      r.add(hcut.data(), cut.p, 2 * (size_t)nnet);
      r.add(hctl, ctl.p, F_WORDS);
      r.add(&herr, err.p);
      r.wait();
    }
    if (herr & DEV_ERR_TIMEOUT) fail(CDS_ERR_TIMEOUT, "push-relabel: device iteration budget exhausted");
    if (herr) fail(CDS_ERR_CUDA, "push-relabel: device error");
    const bool stopped = hctl[F_STOPPED] != 0;
    if (stopped) ans.early_stopped = 1;
    if (c->prof) {
      // cycles (global relabel + rounds) and BFS levels of this max-flow
      std::lock_guard<std::mutex> g(c->mu);
      auto &a = c->prof_done["flow_cycles"];
      a.first += 1;
      a.second += hctl[F_CYCLES];
      auto &b = c->prof_done["flow_bfs_levels"];
      b.first += 1;
      b.second += hctl[F_BFS];
      auto &r = c->prof_done["flow_rounds"];
      r.first += 1;
      r.second += hctl[F_ROUNDS];
      unsigned long long hph[5];
      {
        HostReads r(s);
        r.add(hph, phase.p, 5);
        r.wait();
      }
      CDS_CUDA(cudaMemsetAsync(phase.p, 0, sizeof(hph), s));
      static const char *pn[5] = {"flow_phase_bfs", "flow_phase_check", "flow_phase_prepare",
                                  "flow_phase_push", "flow_phase_relabel"};
      for (int i = 0; i < 5; i++) {
        auto &a2 = c->prof_done[pn[i]];
        a2.first += 1;
        a2.second += hph[i] / 1e6;
      }
    }
    ans.flows++;
    // decide every open network
    bool any_fin = false;
    for (uint32_t i = 0; i < nnet; i++) {
      hfin[i] = 0;
      if (!hact[i]) continue;
      CompState &cs = st[i];
      const int64_t mci = (int64_t)(co.comp_cbeg[i + 1] - co.comp_cbeg[i]);
      const bool saturated = hsink[i] == (long long)hQ[i] * (long long)k * mci;
      const int64_t sz = (int64_t)hcut[i], cnt = (int64_t)hcut[nnet + i];
      if (saturated) {
        if (cs.certify) {
          cs.done = true;
          ncand--;
          if (cs.improved) {
            // the unreachable side at alpha = rho* is the maximal densest set
            if (sz == 0 || (__int128)cnt * cs.lb_d != (__int128)cs.lb_n * sz)
              fail(CDS_ERR_CUDA, "flow certificate does not match the found density");
            cs.lb_n = cnt;
            cs.lb_d = sz;
            hfin[i] = 1;
            any_fin = true;
          }
        } else {
          cs.ub_n = cs.an;
          cs.ub_d = cs.ad;
        }
      } else if (sz > 0 && frac_lt(cs.an, cs.ad, cnt, sz)) {
        cs.lb_n = cnt;
        cs.lb_d = sz;
        cs.improved = true;
      } else if (stopped) {
        // the flow was cut short and found nothing denser: keep what we have
        cs.done = true;
        cs.cut_short = true;
        ncand--;
        if (cs.improved) {
          hfin[i] = 1;
          any_fin = true;
        }
      } else {
        fail(CDS_ERR_CUDA, "flow cut is not denser than alpha");
      }
    }
    if (any_fin) {
      CDS_CUDA(cudaMemcpyAsync(fin.p, hfin.data(), nnet, cudaMemcpyHostToDevice, s));
      k_mark_answer<<<G, 256, 0, s>>>(p, fin.p, mark.p);
      count_launch();
      CDS_CUDA(cudaGetLastError());
    }
    if (stopped) {
      // sets from an early-stopped flow are only as good as that flow
      for (uint32_t i = 0; i < nnet; i++)
        if (hact[i] && !st[i].done && st[i].improved && !hfin[i]) {
          // keep iterating: the next flow starts from the improved bound
        }
    }
  }

  // per instance: the starting component, or the first component (in order)
  // whose search found a strictly denser set
  std::vector<int32_t> win(ninst, -1);
  for (uint32_t i = 0; i < nnet; i++) {
    const CompState &cs = st[i];
    if (!cs.candidate || !cs.improved) continue;
    const uint32_t in = co.comp_inst[i];
    if (frac_lt(best_n[in], best_d[in], cs.lb_n, cs.lb_d)) {
      best_n[in] = cs.lb_n;
      best_d[in] = cs.lb_d;
      best_comp[in] = (int32_t)i;
      best_is_whole[in] = false;
    }
  }
  // proven upper bound of every instance's optimum: the answer, unless a
  // component's search was cut short (early stop), whose optimum is then
  // bounded only by its last bound (largest core inside, or a saturated probe)
  for (uint32_t in = 0; in < ninst; in++) {
    ans.ub_num[in] = best_comp[in] >= 0 ? (uint64_t)best_n[in] : 0;
    ans.ub_den[in] = best_comp[in] >= 0 ? (uint64_t)best_d[in] : 1;
  }
  for (uint32_t i = 0; i < nnet; i++) {
    const CompState &cs = st[i];
    if (!cs.candidate || !ans.early_stopped) continue;
    const bool certified = cs.done && cs.certify && !cs.cut_short;
    if (certified) continue;
    const uint32_t in = co.comp_inst[i];
    if (frac_lt((int64_t)ans.ub_num[in], (int64_t)ans.ub_den[in], cs.ub_n, cs.ub_d)) {
      ans.ub_num[in] = (uint64_t)cs.ub_n;
      ans.ub_den[in] = (uint64_t)cs.ub_d;
    }
  }
  // gather the answer sets: whole components or marked vertices
  std::vector<uint8_t> want(nnet, 0);
  for (uint32_t in = 0; in < ninst; in++) {
    ans.num[in] = best_comp[in] >= 0 ? (uint64_t)best_n[in] : 0;
    ans.den[in] = best_comp[in] >= 0 ? (uint64_t)best_d[in] : 0;
    if (best_comp[in] >= 0) want[best_comp[in]] = 1;
  }
  {
    // whole components: mark every vertex
    std::vector<uint8_t> whole(nnet, 0);
    bool anyw = false;
    for (uint32_t in = 0; in < ninst; in++)
      if (best_comp[in] >= 0 && best_is_whole[in]) {
        whole[best_comp[in]] = 1;
        anyw = true;
      }
    if (anyw) {
      CDS_CUDA(cudaMemcpyAsync(fin.p, whole.data(), nnet, cudaMemcpyHostToDevice, s));
      // a whole component: every vertex is in the answer
      std::vector<uint32_t> tmp;
      for (uint32_t i = 0; i < nnet; i++)
        if (whole[i])
          CDS_CUDA(cudaMemsetAsync(mark.p + co.comp_vbeg[i], 1, co.comp_vbeg[i + 1] - co.comp_vbeg[i], s));
    }
  }
  DBuf<uint8_t> dwant(c, s, nnet);
  CDS_CUDA(cudaMemcpyAsync(dwant.p, want.data(), nnet, cudaMemcpyHostToDevice, s));
  DBuf<uint32_t> outv(c, s, nv + 1), cnt(c, s, 1);
  cnt.zero();
  k_collect<<<G, 256, 0, s>>>(mark.p, co.vcnet.p, co.vmap.p, nv, dwant.p, outv.p, cnt.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  const uint32_t total = d2h(cnt.p, s);
  std::vector<uint32_t> hv_out(total);
  if (total) {
    HostReads r(s);
    r.add(hv_out.data(), outv.p, total);
    r.wait();
  }
  // split per instance (vertex ids are union ids; instances own id ranges)
  std::sort(hv_out.begin(), hv_out.end());
  for (uint32_t v : hv_out) {
    const uint32_t in =
        (uint32_t)(std::upper_bound(inst.h_vbeg.begin(), inst.h_vbeg.end(), v) - inst.h_vbeg.begin()) - 1;
    ans.set[in].push_back(v - inst.h_vbeg[in]);
  }
  for (uint32_t in = 0; in < ninst; in++)
    if (ans.set[in].size() != ans.den[in])
      fail(CDS_ERR_CUDA, "answer set size does not match its density denominator");
}

}  // namespace cds
