// peel.cu -- (k,Psi)-clique-core decomposition.
//
// Replaces cliqueCoreDecompose (cudaCode/main.cu:252-343) with selectNodes /
// processNodesByWarp (cudaCode/src/helpers.cu:611-750), whose removal step
// scans every clique for each removed vertex, and the serial oracle's peel
// (cpuCode/c++/src/helpers.cpp:16-150).
//
// One persistent cooperative kernel runs the whole peel.  Level l has a
// threshold L_l and an alive list A_l (every vertex of the L_l-core, plus
// vertices removed since the list was built).
//   START    block 0 applies the last level's removals to the per-instance
//            counters and compares each instance's alive density with its
//            best (RECORD); the alive set is the L_l-core.
//   COLLECT  each alive vertex of A_l with degree <= L_l gets core number
//            L_l and enters the removal buffer as tasks of up to `chunk`
//            incidences; every other alive vertex enters A_{l+1}, and its
//            degree enters the running minimum M_{l+1}.
//   PROCESS  warps take tasks from the removal buffer; each incident clique
//            not yet retired is retired (atomicOr on a bitmask) and its other
//            members lose one clique each (warp-aggregated atomicSub); a
//            member whose degree crosses L_l is removed at level L_l and its
//            tasks join the same buffer; a member that stays above L_l puts
//            its new degree into M_{l+1}.
// The level ends when every block has collected and no task is outstanding;
// each block sees that by itself and starts level l+1 with L_{l+1} = M_{l+1},
// so a level costs one termination check and no grid barrier.  M_{l+1} is the
// minimum alive degree, or smaller when a vertex entered it and was removed
// later in the same level; the next level then removes nothing and computes
// the exact minimum, so core numbers are unchanged.  Counters rotate over
// four sets, so the set a level uses was cleared two levels before by block 0
// when no block could still read it.  Tasks carry their level's tag, so a
// warp that lags behind the end of a level never takes a next-level task.
// Work is O(k|Psi|) incidence reads in total.  Every wait is bounded; the
// kernel leaves with DEV_ERR_TIMEOUT instead of hanging.
#include "device_util.cuh"
#include "stages.h"

#include <algorithm>
#include <cooperative_groups.h>

namespace {

constexpr uint32_t UNSET = 0xFFFFFFFFu;

struct PeelParams {
  uint32_t n, k;
  uint64_t m;
  const uint32_t *members;      // [m*k]
  const uint64_t *inc_off;      // [n+1]
  const uint32_t *inc;          // [k*m] clique ids
  uint32_t *deg;                // [n] current clique degree
  uint32_t *core;               // [n] UNSET while alive
  uint32_t *retired;            // [(m+31)/32] bitmask
  uint32_t *alive[2];           // alive lists, by level parity
  unsigned long long *queue;    // removal buffer: (v + 1) << 32 | tag << 28 | chunk, 0 = empty
  uint64_t task_cap;
  uint32_t chunk;
  const uint32_t *of_vertex;    // instance of each vertex (null: one instance)
  uint32_t ninst;
  uint32_t *inst_alive_v;               // [ninst] alive vertices at the last RECORD
  unsigned long long *inst_alive_c;     // [ninst] alive cliques at the last RECORD
  uint32_t *inst_pending[2];            // [ninst] removals of the levels of each parity
  unsigned long long *inst_retired[2];  // [ninst] cliques retired likewise
  unsigned long long *best_num; // [ninst]
  unsigned long long *best_den; // [ninst]
  uint32_t *ctl;                // four counter sets, then CTL_LEVELS
  uint32_t *err;
  unsigned long long spin_limit;
  uint64_t max_steps;
  unsigned long long time_budget_ns;  // wall-clock budget of the whole kernel
  unsigned long long *phase_ns;       // [8] block 0's time per phase, summed (profiling)
};

// One counter set per level (level l uses set l & 3), each hot counter on its
// own 128-byte line.
enum {
  S_ACNT = 0,    // size of this level's alive list, filled by the level before
  S_MIN = 32,    // this level's threshold, the running minimum of the level before
  S_HEAD = 64,   // removal buffer: next slot to take
  S_TAIL = 96,   //                 next slot to fill
  S_OUT = 128,   //                 tasks filled but not finished
  S_CDONE = 160, //                 blocks done with COLLECT
  S_REM = 192,   // nonzero once this level removed a vertex
  SET_WORDS = 256,
  CTL_LEVELS = 4 * SET_WORDS,  // levels that removed a vertex
  CTL_STEPS = CTL_LEVELS + 1,  // levels run
  CTL_WORDS = CTL_LEVELS + 32
};
constexpr uint32_t TAG_SHIFT = 28;
constexpr uint32_t CHUNK_MASK = (1u << TAG_SHIFT) - 1u;

__device__ __forceinline__ uint32_t inst_of(const PeelParams &p, uint32_t v) {
  return p.of_vertex ? p.of_vertex[v] : 0u;
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *a) {
  return *(const volatile uint32_t *)a;
}

// Appends the tasks of vertex v (all its incidences, `chunk` at a time) to
// the removal buffer; called by all 32 lanes of a warp with the same v.  The
// outstanding count rises first; each writing lane fences before its stores,
// so a thread that acquires a slot also sees the count (tasks may then only
// finish after they were counted).
__device__ __forceinline__ void push_tasks_warp(const PeelParams &p, uint32_t *set, uint32_t tag,
                                                uint32_t v) {
  const uint64_t len = p.inc_off[v + 1] - p.inc_off[v];
  if (!len) return;
  const uint32_t nt = (uint32_t)((len + p.chunk - 1) / p.chunk);
  uint32_t at = 0;
  if (lane_id() == 0) {
    atomicAdd(set + S_OUT, nt);
    at = atomicAdd(set + S_TAIL, nt);
  }
  at = __shfl_sync(CDS_FULL, at, 0);
  if ((uint64_t)at + nt > p.task_cap) {
    if (lane_id() == 0) atomicOr(p.err, DEV_ERR_OVERFLOW);
    return;
  }
  __syncwarp();
  if (lane_id() < nt) __threadfence();
  const unsigned long long hi = ((unsigned long long)(v + 1) << 32) | ((unsigned long long)tag << TAG_SHIFT);
  for (uint32_t t = lane_id(); t < nt; t += 32)
    *(volatile unsigned long long *)&p.queue[at + t] = hi | t;
}

// The members w of the just-retired cliques (UNSET where a lane has none)
// lose one clique each.  A member crossing L is claimed for level L (a COLLECT
// of another block may claim it first) and its tasks are pushed; a member
// staying above L lowers *tmin to its new degree.  All 32 lanes call it.
__device__ __forceinline__ void drop_members(const PeelParams &p, uint32_t *set, uint32_t tag,
                                             uint32_t par, uint32_t L, const uint32_t *w,
                                             int cnt_members, uint32_t &tmin) {
  constexpr int MAXW = 6;
  uint32_t old[MAXW], cnt[MAXW];
  bool lead[MAXW];
#pragma unroll
  for (int j = 0; j < MAXW; j++) {
    lead[j] = false;
    old[j] = 0;
    cnt[j] = 0;
    if (j < cnt_members) {
      const uint32_t grp = __match_any_sync(CDS_FULL, w[j]);
      lead[j] = w[j] != UNSET && (__ffs(grp) - 1) == (int)lane_id();
      cnt[j] = __popc(grp);
      if (lead[j]) old[j] = atomicSub(&p.deg[w[j]], cnt[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < MAXW; j++) {
    if (j >= cnt_members) break;
    bool drop = false;
    if (lead[j] && old[j] > L) {
      const uint32_t nv = old[j] - cnt[j];
      if (nv > L) {
        tmin = nv < tmin ? nv : tmin;
      } else if (atomicCAS(&p.core[w[j]], UNSET, L) == UNSET) {
        atomicAdd(&p.inst_pending[par][inst_of(p, w[j])], 1u);
        drop = true;
      }
    }
    uint32_t todo = __ballot_sync(CDS_FULL, drop);
    while (todo) {
      const int src_lane = __ffs(todo) - 1;
      todo &= todo - 1;
      push_tasks_warp(p, set, tag, __shfl_sync(CDS_FULL, w[j], src_lane));
    }
  }
}

// K > 0 (2..6): clique size known at compile time, all members loaded
// together; K == 0: any k, six members at a time.
template <int K>
__global__ void __launch_bounds__(1024, 1) k_peel(PeelParams p) {
  __shared__ uint32_t s_min, s_rem, s_nalive, s_L, s_err;
  __shared__ volatile uint32_t s_tail, s_done, s_head;
  const uint32_t k = K ? K : p.k;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  bool done = false;
  const unsigned long long t0 = globaltimer_ns();
  unsigned long long tp = t0;
  unsigned long long acc[3] = {0, 0, 0};
  uint64_t tasks = 0;
#define PHASE(i)                                       \
  do {                                                 \
    if (p.phase_ns && threadIdx.x == 0) {              \
      const unsigned long long now = globaltimer_ns(); \
      acc[i] += now - tp;                              \
      tp = now;                                        \
    }                                                  \
  } while (0)
  for (uint64_t level = 0; level < p.max_steps; level++) {
    uint32_t *set = p.ctl + (level & 3) * SET_WORDS;
    uint32_t *nset = p.ctl + ((level + 1) & 3) * SET_WORDS;
    const uint32_t par = level & 1u;
    const uint32_t tag = level & 3u;
    // ---------------- START ----------------
    // Block 0 began this level after every block had finished level l-2 and
    // collected level l-1, so set (l+2)&3 -- last used by level l-2 -- is
    // free; it is cleared before block 0 signals its COLLECT of this level,
    // hence before any block can reach level l+1, the first to fill it.
    if (blockIdx.x == 0) {
      if (threadIdx.x == 0) {
        if (globaltimer_ns() - t0 > p.time_budget_ns) atomicOr(p.err, DEV_ERR_TIMEOUT);
        uint32_t *fset = p.ctl + ((level + 2) & 3) * SET_WORDS;
        fset[S_ACNT] = 0;
        fset[S_MIN] = UNSET;
        fset[S_HEAD] = 0;
        fset[S_TAIL] = 0;
        fset[S_OUT] = 0;
        fset[S_CDONE] = 0;
        fset[S_REM] = 0;
        if (level > 0 && ld_volatile(p.ctl + ((level + 3) & 3) * SET_WORDS + S_REM))
          p.ctl[CTL_LEVELS] += 1;
        p.ctl[CTL_STEPS] += 1;
      }
      // RECORD: the removals of level l-1 are complete; the alive set is this
      // level's core
      const uint32_t q = par ^ 1u;
      for (uint32_t i = threadIdx.x; i < p.ninst; i += blockDim.x) {
        const uint32_t av = p.inst_alive_v[i] - __ldcg(p.inst_pending[q] + i);
        const unsigned long long ac = p.inst_alive_c[i] - __ldcg(p.inst_retired[q] + i);
        p.inst_pending[q][i] = 0;
        p.inst_retired[q][i] = 0;
        p.inst_alive_v[i] = av;
        p.inst_alive_c[i] = ac;
        if (!av) continue;
        const unsigned long long bn = p.best_num[i], bd = p.best_den[i];
        // ac/av > bn/bd  <=>  ac*bd > bn*av  (128-bit products)
        const unsigned long long lh = __umul64hi(ac, bd), ll = ac * bd;
        const unsigned long long rh = __umul64hi(bn, (unsigned long long)av), rl = bn * av;
        if (bd == 0 || lh > rh || (lh == rh && ll > rl)) {
          p.best_num[i] = ac;
          p.best_den[i] = av;
        }
      }
    }
    if (threadIdx.x == 0) {
      s_nalive = ld_volatile(set + S_ACNT);
      s_L = ld_volatile(set + S_MIN);
      s_err = ld_volatile(p.err);
      s_min = UNSET;
      s_rem = 0;
      s_tail = 0;
      s_done = 0;
      s_head = 0;
    }
    __syncthreads();
    if (s_err) return;
    const uint32_t nalive = s_nalive;
    if (nalive == 0) {
      done = true;
      break;
    }
    const uint32_t L = s_L;
    if (L == UNSET) {  // survivors always bring their degree into the minimum
      if (threadIdx.x == 0) atomicOr(p.err, DEV_ERR_INTERNAL);
      return;
    }
    PHASE(0);
    // ---------------- COLLECT ----------------
    const uint32_t *src = p.alive[par];
    uint32_t *dst = p.alive[par ^ 1u];
    uint32_t my_min = UNSET;
    bool any_rm = false;
    for (uint32_t base = gwarp * 32; base < nalive; base += nwarps * 32) {
      const uint32_t i = base + lane;
      uint32_t v = 0, d = 0;
      bool rm = false, keep = false;
      if (i < nalive) {
        // L2 loads: other blocks wrote these during the last level
        v = level == 0 ? i : __ldcg(src + i);
        if (__ldcg(p.core + v) == UNSET) {
          d = __ldcg(p.deg + v);
          // claim: a PROCESS warp of a faster block may remove v first
          if (d <= L)
            rm = atomicCAS(&p.core[v], UNSET, L) == UNSET;
          else
            keep = true;
        }
      }
      const uint32_t km = __ballot_sync(CDS_FULL, keep);
      if (km) {
        uint32_t at = 0;
        if (lane == 0) at = atomicAdd(nset + S_ACNT, (uint32_t)__popc(km));
        at = __shfl_sync(CDS_FULL, at, 0);
        if (keep) {
          dst[at + __popc(km & ((1u << lane) - 1u))] = v;
          my_min = d < my_min ? d : my_min;
        }
      }
      uint32_t todo = __ballot_sync(CDS_FULL, rm);
      if (todo) {
        any_rm = true;
        agg_inc(p.inst_pending[par], rm ? inst_of(p, v) : 0u, rm);
        while (todo) {
          const int src_lane = __ffs(todo) - 1;
          todo &= todo - 1;
          push_tasks_warp(p, set, tag, __shfl_sync(CDS_FULL, v, src_lane));
        }
      }
    }
    my_min = warp_min(my_min);
    if (lane == 0) {
      if (my_min != UNSET) atomicMin(&s_min, my_min);
      if (any_rm) s_rem = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // release: the block's pushes and minimum come first
      if (s_min != UNSET) atomicMin(nset + S_MIN, s_min);
      if (s_rem) atomicOr(set + S_REM, 1u);
      atom_add_release(set + S_CDONE, 1u);
    }
    PHASE(1);
    // Drain the removal buffer.  Warp 0 of each block is a dispatcher: it
    // alone polls the global tail and the end of the level (every block has
    // collected and no task is outstanding; tasks are only added while
    // another task is in hand) and publishes both in shared memory.  The
    // other warps read shared memory while idle, take slots in order and
    // wait for a taken slot to be filled.
    if ((threadIdx.x >> 5) == 0) {
      if (lane == 0) {
        unsigned long long spins = 0;
        unsigned int ns = 32;
        for (;;) {
          s_tail = ld_volatile(set + S_TAIL);
          if (ld_acquire(set + S_CDONE) == gridDim.x && ld_acquire(set + S_OUT) == 0) break;
          if (ld_volatile(p.err)) break;
          if (++spins > p.spin_limit) {
            atomicOr(p.err, DEV_ERR_TIMEOUT);
            break;
          }
          __nanosleep(ns);
          if (ns < 128) ns <<= 1;
        }
        s_done = 1;
      }
      __syncwarp();
    }
    for (;;) {
      if ((threadIdx.x >> 5) == 0) break;
      unsigned long long task = 0;
      int state = 0;  // 0 wait, 1 task, 2 drained
      if (lane == 0) {
        bool have = false;
        uint32_t h = 0;
        unsigned long long spins = 0;
        for (;;) {
          const uint32_t done_now = s_done;
          if (!have && s_head < s_tail) {
            h = atomicAdd(set + S_HEAD, 1u);
            atomicMax((uint32_t *)&s_head, h + 1);
            have = true;
          }
          if (have && h < p.task_cap) {
            task = ld_acquire_u64(&p.queue[h]);
            // a task of the next level is not ours: that level began after
            // this one ended, which the dispatcher is about to see
            if (task && ((uint32_t)task >> TAG_SHIFT) == tag) {
              p.queue[h] = 0;
              state = 1;
              break;
            }
          }
          // drained: nothing was published before the dispatcher saw the end
          if (done_now) {
            state = 2;
            break;
          }
          if (++spins > p.spin_limit) {
            atomicOr(p.err, DEV_ERR_TIMEOUT);
            state = 2;
            break;
          }
          __nanosleep(32);
        }
      }
      state = __shfl_sync(CDS_FULL, state, 0);
      if (state == 2) break;
      task = __shfl_sync(CDS_FULL, task, 0);
      const uint32_t v = (uint32_t)(task >> 32) - 1u;
      const uint64_t b = p.inc_off[v] + (uint64_t)((uint32_t)task & CHUNK_MASK) * p.chunk;
      const uint64_t e = min(b + p.chunk, p.inc_off[v + 1]);
      const uint32_t vi = inst_of(p, v);
      uint32_t tmin = UNSET;
      for (uint64_t i0 = b; i0 < e; i0 += 32) {
        const uint64_t i = i0 + lane;
        uint32_t c = 0;
        bool mine = false;
        if (i < e) {
          c = p.inc[i];
          const uint32_t bit = 1u << (c & 31);
          mine = !(atomicOr(&p.retired[c >> 5], bit) & bit);
        }
        const uint32_t won = __ballot_sync(CDS_FULL, mine);
        if (!won) continue;
        if (lane == 0) atomicAdd(&p.inst_retired[par][vi], (unsigned long long)__popc(won));
        if (K > 0) {
          // the k members, loaded together (v's own slot passes as UNSET)
          uint32_t w[K > 0 ? K : 1];
#pragma unroll
          for (int j = 0; j < K; j++) {
            uint32_t x = UNSET;
            if (mine) {
              x = p.members[(uint64_t)c * K + j];
              if (x == v) x = UNSET;
            }
            w[j] = x;
          }
          drop_members(p, set, tag, par, L, w, K, tmin);
        } else {
          for (uint32_t j0 = 0; j0 < k; j0 += 6) {
            uint32_t w[6];
            const int nw = (int)min(6u, k - j0);
#pragma unroll
            for (int j = 0; j < 6; j++) {
              uint32_t x = UNSET;
              if (j < nw && mine) {
                x = p.members[(uint64_t)c * k + j0 + j];
                if (x == v) x = UNSET;
              }
              w[j] = x;
            }
            drop_members(p, set, tag, par, L, w, nw, tmin);
          }
        }
      }
      tmin = warp_min(tmin);
      if (lane == 0) {
        if (tmin != UNSET) atomicMin(nset + S_MIN, tmin);
        // release: the tasks this one pushed and its minimum come first
        atom_add_release(set + S_OUT, 0xFFFFFFFFu);
      }
      __syncwarp();
    }
    __syncthreads();
    PHASE(2);
    if (p.phase_ns && threadIdx.x == 0) tasks += ld_volatile(set + S_TAIL);
  }
#undef PHASE
  if (p.phase_ns && blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < 3; i++) p.phase_ns[i] = acc[i];
    p.phase_ns[3] = tasks;
  }
  if (!done && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(p.err, DEV_ERR_TIMEOUT);  // level budget exhausted
}

// incidence lists: slot j of clique c goes to members[c*k+j]'s list
__global__ void k_fill_incidence(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                                 const uint64_t *__restrict__ inc_off, uint32_t *__restrict__ cursor,
                                 uint32_t *__restrict__ inc) {
  const uint64_t total = m * k;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
    const uint64_t t = base + threadIdx.x;
    // slot-major order: lanes see the same slot of consecutive cliques, which
    // share their root, so the cursor atomics aggregate
    const bool ok = t < total;
    uint32_t v = UNSET, c = 0;
    if (ok) {
      const uint64_t j = t / m;
      c = (uint32_t)(t - j * m);
      v = members[(uint64_t)c * k + j];
    }
    const uint32_t grp = __match_any_sync(CDS_FULL, v);
    const uint32_t leader = __ffs(grp) - 1;
    uint32_t at = 0;
    if (ok && leader == lane_id()) at = atomicAdd(&cursor[v], (uint32_t)__popc(grp));
    at = __shfl_sync(grp, at, leader);
    if (ok) inc[inc_off[v] + at + __popc(grp & ((1u << lane_id()) - 1u))] = c;
  }
}

__global__ void k_inst_cliques(const uint32_t *__restrict__ members, uint64_t m, uint32_t k,
                               const uint32_t *__restrict__ of_vertex,
                               unsigned long long *__restrict__ alive_c) {
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m;
       c += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&alive_c[of_vertex[members[c * k]]], 1ull);
}

__global__ void k_inst_maxcore(const uint32_t *__restrict__ core, uint32_t n,
                               const uint32_t *__restrict__ of_vertex, uint32_t *__restrict__ out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    atomicMax(&out[of_vertex ? of_vertex[v] : 0u], core[v]);
}

// the first level's threshold: the minimum clique degree
__global__ void k_min_degree(const uint32_t *__restrict__ deg, uint32_t n, uint32_t *__restrict__ out) {
  uint32_t m = UNSET;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    m = min(m, deg[v]);
  m = warp_min(m);
  if (lane_id() == 0 && m != UNSET) atomicMin(out, m);
}

}  // namespace

namespace cds {

void peel(cds_ctx *c, cudaStream_t s, uint32_t n, const Cliques &cl, const Instances &inst,
          const Tuning &t, uint32_t gl_buffer_size, PeelOut &out) {
  const uint32_t k = cl.k;
  const uint64_t m = cl.count;
  const uint32_t ninst = inst.count;
  out.core.c = c;
  out.core.s = s;
  out.core.alloc(n + 1);
  out.best_num.assign(ninst, 0);
  out.best_den.assign(ninst, 0);
  out.inst_max_core.assign(ninst, 0);
  if (n == 0) return;

  // vertex -> clique incidence CSR
  DBuf<uint64_t> inc_off(c, s, n + 1);
  scan_u32(cl.cdeg.p, inc_off.p, n, c, s);
  DBuf<uint32_t> inc(c, s, m * k + 1);
  {
    DBuf<uint32_t> cursor(c, s, n);
    cursor.zero();
    if (m) {
      ProfScope ps(c, s, "peel_incidence");
      k_fill_incidence<<<c->sm_count * 8, 256, 0, s>>>(cl.members.p, m, k, inc_off.p, cursor.p,
                                                      inc.p);
      count_launch();
      CDS_CUDA(cudaGetLastError());
    }
  }

  // Removal-buffer tasks are short (t.peel_chunk incidences) so that a level's
  // work, above all a hub's incidence list, spreads over many warps; the
  // reference's glBufferSize (a per-block buffer length) has no role here,
  // the buffer being sized exactly from the incidence counts.
  (void)gl_buffer_size;
  const uint32_t chunk = (uint32_t)std::max(32, std::min(t.peel_chunk, 1 << 16));
  const uint64_t task_cap = (uint64_t)n + (m * k) / chunk + 64;
  if (task_cap >= 0xFFFFFFFFull) fail(CDS_ERR_OVERFLOW, "removal buffer exceeds 32-bit indexing");
  DBuf<uint32_t> deg(c, s, n);
  CDS_CUDA(cudaMemcpyAsync(deg.p, cl.cdeg.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  CDS_CUDA(cudaMemsetAsync(out.core.p, 0xFF, (size_t)n * 4, s));
  DBuf<uint32_t> retired(c, s, (m + 31) / 32 + 1);
  retired.zero();
  DBuf<uint32_t> alive(c, s, 2 * (size_t)n);
  DBuf<unsigned long long> queue(c, s, task_cap);
  queue.zero();
  // per-instance counters
  DBuf<uint32_t> ia_v(c, s, ninst), ipend(c, s, 2 * (size_t)ninst);
  DBuf<unsigned long long> ia_c(c, s, ninst), iret(c, s, 2 * (size_t)ninst), bnum(c, s, ninst),
      bden(c, s, ninst);
  {
    std::vector<uint32_t> hv(ninst);
    for (uint32_t i = 0; i < ninst; i++) hv[i] = inst.h_vbeg[i + 1] - inst.h_vbeg[i];
    CDS_CUDA(cudaMemcpyAsync(ia_v.p, hv.data(), ninst * 4, cudaMemcpyHostToDevice, s));
    CDS_CUDA(cudaStreamSynchronize(s));
  }
  ipend.zero();
  iret.zero();
  bnum.zero();
  bden.zero();
  if (ninst == 1) {
    const unsigned long long mm = m;
    CDS_CUDA(cudaMemcpyAsync(ia_c.p, &mm, 8, cudaMemcpyHostToDevice, s));
    CDS_CUDA(cudaStreamSynchronize(s));
  } else {
    ia_c.zero();
    if (m) {
      k_inst_cliques<<<c->sm_count * 4, 256, 0, s>>>(cl.members.p, m, k, inst.of_vertex.p, ia_c.p);
      count_launch();
    }
  }
  // counter sets: set 0 holds the first level (all n vertices, threshold the
  // minimum degree), the others start empty with an unset minimum
  DBuf<uint32_t> ctl(c, s, CTL_WORDS);
  DBuf<uint32_t> err(c, s, 1);
  err.zero();
  {
    std::vector<uint32_t> init(CTL_WORDS, 0);
    for (int i = 0; i < 4; i++) init[i * SET_WORDS + S_MIN] = UNSET;
    init[S_ACNT] = n;
    CDS_CUDA(cudaMemcpyAsync(ctl.p, init.data(), CTL_WORDS * 4, cudaMemcpyHostToDevice, s));
    k_min_degree<<<c->sm_count * 2, 256, 0, s>>>(deg.p, n, ctl.p + S_MIN);
    count_launch();
    CDS_CUDA(cudaGetLastError());
    CDS_CUDA(cudaStreamSynchronize(s));
  }

  PeelParams p{};
  p.n = n;
  p.k = k;
  p.m = m;
  p.members = cl.members.p;
  p.inc_off = inc_off.p;
  p.inc = inc.p;
  p.deg = deg.p;
  p.core = out.core.p;
  p.retired = retired.p;
  p.alive[0] = alive.p;
  p.alive[1] = alive.p + n;
  p.queue = queue.p;
  p.task_cap = task_cap;
  p.chunk = chunk;
  p.of_vertex = ninst > 1 ? inst.of_vertex.p : nullptr;
  p.ninst = ninst;
  p.inst_alive_v = ia_v.p;
  p.inst_alive_c = ia_c.p;
  p.inst_pending[0] = ipend.p;
  p.inst_pending[1] = ipend.p + ninst;
  p.inst_retired[0] = iret.p;
  p.inst_retired[1] = iret.p + ninst;
  p.best_num = bnum.p;
  p.best_den = bden.p;
  p.ctl = ctl.p;
  p.err = err.p;
  p.spin_limit = 1ull << 24;
  p.max_steps = 4ull * n + 16;
  p.time_budget_ns = 120ull * 1000000000ull;
  DBuf<unsigned long long> phase(c, s, 8);
  phase.zero();
  p.phase_ns = c->prof ? phase.p : nullptr;

  const int threads = 1024;
  void *kern = k == 2 ? (void *)k_peel<2>
             : k == 3 ? (void *)k_peel<3>
             : k == 4 ? (void *)k_peel<4>
             : k == 5 ? (void *)k_peel<5>
             : k == 6 ? (void *)k_peel<6>
                      : (void *)k_peel<0>;
  int per_sm = 0;
  CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0));
  if (per_sm < 1) fail(CDS_ERR_CUDA, "peel kernel does not fit on an SM");
  per_sm = 1;
  dim3 grid(coop_grid(c, per_sm)), block(threads);
  void *args[] = {&p};
  {
    ProfScope ps(c, s, "peel");
    CDS_CUDA(cudaLaunchCooperativeKernel(kern, grid, block, args, 0, s));
  }
  count_launch();
  CDS_CUDA(cudaGetLastError());

  DBuf<uint32_t> imax(c, s, ninst);
  imax.zero();
  k_inst_maxcore<<<c->sm_count * 4, 256, 0, s>>>(out.core.p, n,
                                                 ninst > 1 ? inst.of_vertex.p : nullptr, imax.p);
  count_launch();
  CDS_CUDA(cudaGetLastError());
  const uint32_t e = d2h(err.p, s);
  if (e & DEV_ERR_TIMEOUT) fail(CDS_ERR_TIMEOUT, "peel: device iteration budget exhausted");
  if (e & DEV_ERR_OVERFLOW) fail(CDS_ERR_OVERFLOW, "peel: removal buffer overflow");
  if (e & DEV_ERR_INTERNAL) fail(CDS_ERR_CUDA, "peel: internal invariant failed");
  if (e) fail(CDS_ERR_CUDA, "peel: device error");
  std::vector<unsigned long long> hn(ninst), hd(ninst);
  CDS_CUDA(cudaMemcpyAsync(hn.data(), bnum.p, ninst * 8, cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaMemcpyAsync(hd.data(), bden.p, ninst * 8, cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaMemcpyAsync(out.inst_max_core.data(), imax.p, ninst * 4, cudaMemcpyDeviceToHost, s));
  uint32_t levels[2] = {0, 0};
  CDS_CUDA(cudaMemcpyAsync(levels, ctl.p + CTL_LEVELS, 8, cudaMemcpyDeviceToHost, s));
  unsigned long long hph[8] = {0};
  if (c->prof) CDS_CUDA(cudaMemcpyAsync(hph, phase.p, sizeof(hph), cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaStreamSynchronize(s));
  if (c->prof) {
    // phase breakdown of block 0 (ms), the removal-buffer task count and the
    // levels run (those that removed nothing included)
    static const char *names[5] = {"peel_phase_start", "peel_phase_collect", "peel_phase_drain",
                                   "peel_tasks_x1e-6", "peel_steps_x1e-6"};
    hph[4] = levels[1];
    std::lock_guard<std::mutex> g(c->mu);
    for (int i = 0; i < 5; i++) {
      auto &slot = c->prof_done[names[i]];
      slot.first += 1;
      slot.second += hph[i] / 1e6;
    }
  }
  out.levels = levels[0];
  out.max_core = 0;
  for (uint32_t i = 0; i < ninst; i++) {
    out.best_num[i] = hn[i];
    out.best_den[i] = hd[i];
    out.max_core = std::max(out.max_core, out.inst_max_core[i]);
  }
}

}  // namespace cds
