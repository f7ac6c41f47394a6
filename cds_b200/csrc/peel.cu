// peel.cu -- (k,Psi)-clique-core decomposition.
//
// Replaces cliqueCoreDecompose (cudaCode/main.cu:252-343) with selectNodes /
// processNodesByWarp (cudaCode/src/helpers.cu:611-750), whose removal step
// scans every clique for each removed vertex, and the serial oracle's peel
// (cpuCode/c++/src/helpers.cpp:16-150).
//
// One persistent cooperative kernel runs the whole peel.  Each level L:
//   SCAN     compact the alive list and take the minimum clique degree;
//            L = max(L, minimum).  The alive set is the L-core; block 0
//            compares its density with each instance's best (RECORD).
//   COLLECT  every alive vertex with degree <= L gets core number L and
//            enters the removal buffer as tasks of up to `chunk` incidences.
//   PROCESS  warps take tasks from the removal buffer; each incident clique
//            not yet retired is retired (atomicOr on a bitmask) and its other
//            members lose one clique each (warp-aggregated atomicSub); a
//            member whose degree crosses L is removed at level L and its
//            tasks join the same buffer, which drains without further grid
//            barriers.  Two grid barriers per level in all.
// Work is O(k|Psi|) incidence reads in total.  Every wait is a bounded grid
// barrier; the kernel leaves with DEV_ERR_TIMEOUT instead of hanging.
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
  uint32_t *alive[2];           // alive lists
  unsigned long long *queue;    // removal buffer: ((v + 1) << 32 | chunk), 0 = empty slot
  uint64_t task_cap;
  uint32_t chunk;
  const uint32_t *of_vertex;    // instance of each vertex (null: one instance)
  uint32_t ninst;
  uint32_t *inst_alive_v;       // [ninst]
  unsigned long long *inst_alive_c;   // [ninst]
  uint32_t *inst_pending;       // [ninst] removals not yet applied to alive_v
  unsigned long long *best_num; // [ninst]
  unsigned long long *best_den; // [ninst]
  // control block
  uint32_t *ctl;                // see CTL_* below
  GridBarrier *bar;
  uint32_t *err;
  unsigned long long spin_limit;
  uint64_t max_steps;
  unsigned long long time_budget_ns;  // wall-clock budget of the whole kernel
  unsigned long long *phase_ns;       // [6] block 0's time per phase, summed (profiling)
};

// Control words, each hot counter on its own 128-byte line.
enum {
  CTL_MIN = 0,        // [2] atomicMin targets of SCAN, by level parity
  CTL_ACNT = 32,      // [2] alive list sizes (+0, +32)
  CTL_HEAD = 96,      // removal buffer: next slot to take
  CTL_TAIL = 128,     //                 next slot to fill
  CTL_OUT = 160,      //                 tasks filled but not finished
  CTL_CDONE = 192,    //                 blocks done with COLLECT
  CTL_LEVEL = 224,
  CTL_LEVELS = 225,
  CTL_WORDS = 256
};
constexpr int CTL_ACNT_STRIDE = 32;

__device__ __forceinline__ uint32_t inst_of(const PeelParams &p, uint32_t v) {
  return p.of_vertex ? p.of_vertex[v] : 0u;
}

// Appends the tasks of vertex v (all its incidences, `chunk` at a time) to
// the removal buffer; called by all 32 lanes of a warp with the same v.  The
// outstanding count rises first; each writing lane fences before its stores,
// so a thread that acquires a slot also sees the count (tasks may then only
// finish after they were counted).
__device__ __forceinline__ void push_tasks_warp(const PeelParams &p, uint32_t v) {
  const uint64_t len = p.inc_off[v + 1] - p.inc_off[v];
  if (!len) return;
  const uint32_t nt = (uint32_t)((len + p.chunk - 1) / p.chunk);
  uint32_t at = 0;
  if (lane_id() == 0) {
    atomicAdd(&p.ctl[CTL_OUT], nt);
    at = atomicAdd(&p.ctl[CTL_TAIL], nt);
  }
  at = __shfl_sync(CDS_FULL, at, 0);
  if ((uint64_t)at + nt > p.task_cap) {
    if (lane_id() == 0) atomicOr(p.err, DEV_ERR_OVERFLOW);
    return;
  }
  __syncwarp();
  if (lane_id() < nt) __threadfence();
  for (uint32_t t = lane_id(); t < nt; t += 32)
    *(volatile unsigned long long *)&p.queue[at + t] = ((unsigned long long)(v + 1) << 32) | t;
}

__global__ void __launch_bounds__(1024, 1) k_peel(PeelParams p) {
  __shared__ uint32_t s_min;
  __shared__ volatile uint32_t s_tail, s_done, s_head;
  volatile uint32_t *ctl = p.ctl;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gthreads = gridDim.x * blockDim.x;
  const uint32_t gwarp = gtid >> 5, nwarps = gthreads >> 5;
  const uint32_t lane = lane_id();
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  uint32_t L = 0;
  bool done = false;
  const unsigned long long t0 = globaltimer_ns();
  unsigned long long tp = globaltimer_ns();
  unsigned long long acc[5] = {0, 0, 0, 0, 0};
  uint64_t tasks = 0;
#define PHASE(i)                                     \
  do {                                               \
    if (p.phase_ns && threadIdx.x == 0) {            \
      const unsigned long long now = globaltimer_ns(); \
      acc[i] += now - tp;                            \
      tp = now;                                      \
    }                                                \
  } while (0)
  for (uint64_t level = 0; level < p.max_steps; level++) {
    const uint32_t src = level & 1u, dst = src ^ 1u;
    // ---------------- SCAN ----------------
    // Past the time budget the leader flags an error that every block sees
    // at the next barrier, so all leave together.
    if (leader) {
      if (globaltimer_ns() - t0 > p.time_budget_ns) atomicOr(p.err, DEV_ERR_TIMEOUT);
      ctl[CTL_HEAD] = 0;  // the removal buffer drained before the last barrier
      ctl[CTL_TAIL] = 0;
      ctl[CTL_OUT] = 0;
      ctl[CTL_CDONE] = 0;
      ctl[CTL_MIN + dst] = UNSET;  // read during the previous level, written next level
    }
    const bool first = level == 0;
    const uint32_t nsrc = first ? p.n : ctl[CTL_ACNT + CTL_ACNT_STRIDE * src];
    if (threadIdx.x == 0) s_min = UNSET;
    __syncthreads();
    uint32_t my_min = UNSET;
    for (uint32_t base = gwarp * 32; base < nsrc; base += nwarps * 32) {
      const uint32_t i = base + lane;
      uint32_t v = 0;
      bool alive = false;
      if (i < nsrc) {
        v = first ? i : p.alive[src][i];
        alive = p.core[v] == UNSET;
      }
      const uint32_t m = __ballot_sync(CDS_FULL, alive);
      uint32_t at = 0;
      if (lane == 0 && m) at = atomicAdd((uint32_t *)&ctl[CTL_ACNT + CTL_ACNT_STRIDE * dst], (uint32_t)__popc(m));
      at = __shfl_sync(CDS_FULL, at, 0);
      if (alive) {
        p.alive[dst][at + __popc(m & ((1u << lane) - 1u))] = v;
        const uint32_t dv = p.deg[v];
        my_min = dv < my_min ? dv : my_min;
      }
    }
    my_min = warp_min(my_min);
    if (lane == 0 && my_min != UNSET) atomicMin(&s_min, my_min);
    __syncthreads();
    if (threadIdx.x == 0 && s_min != UNSET) atomicMin((uint32_t *)&ctl[CTL_MIN + src], s_min);
    if (blockIdx.x == 0) {
      // RECORD: apply the last level's removals; the alive set is now the
      // next level's core, and nothing changes the counters in this phase
      for (uint32_t i = threadIdx.x; i < p.ninst; i += blockDim.x) {
        const unsigned long long av = p.inst_alive_v[i] - p.inst_pending[i];
        p.inst_alive_v[i] = (uint32_t)av;
        p.inst_pending[i] = 0;
        if (!av) continue;
        const unsigned long long ac = p.inst_alive_c[i];
        const unsigned long long bn = p.best_num[i], bd = p.best_den[i];
        // ac/av > bn/bd  <=>  ac*bd > bn*av  (128-bit products)
        const unsigned long long lh = __umul64hi(ac, bd), ll = ac * bd;
        const unsigned long long rh = __umul64hi(bn, av), rl = bn * av;
        if (bd == 0 || lh > rh || (lh == rh && ll > rl)) {
          p.best_num[i] = ac;
          p.best_den[i] = av;
        }
      }
    }
    if (!grid_sync(p.bar, p.err, p.spin_limit)) return;
    PHASE(0);
    const uint32_t nalive = ctl[CTL_ACNT + CTL_ACNT_STRIDE * dst];
    if (nalive == 0) {
      done = true;
      break;
    }
    const uint32_t gmin = ctl[CTL_MIN + src];
    L = gmin > L ? gmin : L;
    // ---------------- COLLECT + PROCESS ----------------
    if (leader) {
      ctl[CTL_ACNT + CTL_ACNT_STRIDE * src] = 0;  // next filled by the next SCAN
      ctl[CTL_LEVEL] = L;
      ctl[CTL_LEVELS] = ctl[CTL_LEVELS] + 1;
    }
    for (uint32_t base = gwarp * 32; base < nalive; base += nwarps * 32) {
      const uint32_t i = base + lane;
      uint32_t v = 0;
      bool rm = false;
      if (i < nalive) {
        v = p.alive[dst][i];
        // claim: a removal by a PROCESS warp of another block may have
        // happened already in this level; the winner counts and pushes
        rm = p.deg[v] <= L && atomicCAS(&p.core[v], UNSET, L) == UNSET;
      }
      agg_inc(p.inst_pending, rm ? inst_of(p, v) : 0u, rm);
      uint32_t todo = __ballot_sync(CDS_FULL, rm);
      while (todo) {
        const int src_lane = __ffs(todo) - 1;
        todo &= todo - 1;
        push_tasks_warp(p, __shfl_sync(CDS_FULL, v, src_lane));
      }
    }
    __syncthreads();
    if (threadIdx.x == 0)  // release: the block's pushes are counted first
      atom_add_release(p.ctl + CTL_CDONE, 1u);
    PHASE(1);
    // Drain the removal buffer.  Warp 0 of each block is a dispatcher: it
    // alone polls the global tail and the termination condition (every block
    // has collected and no task is outstanding; tasks are only added while
    // another task is in hand) and publishes both in shared memory.  The
    // other warps read shared memory while idle, take slots in order and
    // wait for a taken slot to be filled.
    if (threadIdx.x == 0) {
      s_tail = 0;
      s_done = 0;
      s_head = 0;
    }
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
      if (lane == 0) {
        unsigned long long spins = 0;
        unsigned int ns = 32;
        for (;;) {
          s_tail = ctl[CTL_TAIL];
          if (ld_acquire(p.ctl + CTL_CDONE) == gridDim.x && ld_acquire(p.ctl + CTL_OUT) == 0) break;
          if (*(volatile uint32_t *)p.err) break;
          if (++spins > p.spin_limit) {
            atomicOr(p.err, DEV_ERR_TIMEOUT);
            break;
          }
          __nanosleep(ns);
          if (ns < 256) ns <<= 1;
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
            h = atomicAdd((uint32_t *)&ctl[CTL_HEAD], 1u);
            atomicMax((uint32_t *)&s_head, h + 1);
            have = true;
          }
          if (have && h < p.task_cap) {
            task = ld_acquire_u64(&p.queue[h]);
            if (task) {
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
      const uint64_t b = p.inc_off[v] + (uint64_t)(uint32_t)task * p.chunk;
      const uint64_t e = min(b + p.chunk, p.inc_off[v + 1]);
      const uint32_t vi = inst_of(p, v);
      for (uint64_t i0 = b; i0 < e; i0 += 32) {
        const uint64_t i = i0 + lane;
        uint32_t c = UNSET;
        bool mine = false;
        if (i < e) {
          c = p.inc[i];
          const uint32_t bit = 1u << (c & 31);
          mine = !(atomicOr(&p.retired[c >> 5], bit) & bit);
        }
        const uint32_t won = __ballot_sync(CDS_FULL, mine);
        if (!won) continue;
        if (lane == 0)
          atomicAdd(&p.inst_alive_c[vi], (unsigned long long)(-(long long)__popc(won)));
        for (uint32_t j = 0; j < p.k; j++) {
          uint32_t w = UNSET;
          if (mine) {
            w = p.members[(uint64_t)c * p.k + j];
            if (w == v) w = UNSET;
          }
          if (!__any_sync(CDS_FULL, w != UNSET)) continue;
          const uint32_t grp = __match_any_sync(CDS_FULL, w);
          bool drop = false;
          if (w != UNSET && (__ffs(grp) - 1) == (int)lane) {
            const uint32_t cnt = __popc(grp);
            const uint32_t old = atomicSub(&p.deg[w], cnt);
            // w drops to level L: remove it now, unless a COLLECT claimed it
            if (old > L && old - cnt <= L && atomicCAS(&p.core[w], UNSET, L) == UNSET) {
              atomicAdd(&p.inst_pending[inst_of(p, w)], 1u);
              drop = true;
            }
          }
          uint32_t todo = __ballot_sync(CDS_FULL, drop);
          while (todo) {
            const int src_lane = __ffs(todo) - 1;
            todo &= todo - 1;
            push_tasks_warp(p, __shfl_sync(CDS_FULL, w, src_lane));
          }
        }
      }
      __syncwarp();
      if (lane == 0)  // release: the tasks this one pushed are counted first
        atom_add_release(p.ctl + CTL_OUT, 0xFFFFFFFFu);
    }
    __syncthreads();
    PHASE(2);
    if (p.phase_ns && threadIdx.x == 0) tasks += ctl[CTL_TAIL];
    if (!grid_sync(p.bar, p.err, p.spin_limit)) return;
    PHASE(3);
  }
#undef PHASE
  if (p.phase_ns && blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < 4; i++) p.phase_ns[i] = acc[i];
    p.phase_ns[4] = tasks;
  }
  if (!done && leader) atomicOr(p.err, DEV_ERR_TIMEOUT);  // level budget exhausted
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
  DBuf<uint32_t> ia_v(c, s, ninst), ipend(c, s, ninst);
  DBuf<unsigned long long> ia_c(c, s, ninst), bnum(c, s, ninst), bden(c, s, ninst);
  {
    std::vector<uint32_t> hv(ninst);
    for (uint32_t i = 0; i < ninst; i++) hv[i] = inst.h_vbeg[i + 1] - inst.h_vbeg[i];
    CDS_CUDA(cudaMemcpyAsync(ia_v.p, hv.data(), ninst * 4, cudaMemcpyHostToDevice, s));
    CDS_CUDA(cudaStreamSynchronize(s));
  }
  ipend.zero();
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
  DBuf<uint32_t> ctl(c, s, CTL_WORDS);
  DBuf<GridBarrier> bar(c, s, 1);
  DBuf<uint32_t> err(c, s, 1);
  ctl.zero();
  bar.zero();
  err.zero();
  {
    const uint32_t init[2] = {UNSET, UNSET};
    CDS_CUDA(cudaMemcpyAsync(ctl.p + CTL_MIN, init, 8, cudaMemcpyHostToDevice, s));
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
  p.inst_pending = ipend.p;
  p.best_num = bnum.p;
  p.best_den = bden.p;
  p.ctl = ctl.p;
  p.bar = bar.p;
  p.err = err.p;
  p.spin_limit = 1ull << 24;
  p.max_steps = 4ull * n + 16;
  p.time_budget_ns = 120ull * 1000000000ull;
  DBuf<unsigned long long> phase(c, s, 8);
  phase.zero();
  p.phase_ns = c->prof ? phase.p : nullptr;

  const int threads = 1024;
  int per_sm = 0;
  CDS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel, threads, 0));
  if (per_sm < 1) fail(CDS_ERR_CUDA, "peel kernel does not fit on an SM");
  per_sm = 1;
  dim3 grid(coop_grid(c, per_sm)), block(threads);
  void *args[] = {&p};
  {
    ProfScope ps(c, s, "peel");
    CDS_CUDA(cudaLaunchCooperativeKernel((void *)k_peel, grid, block, args, 0, s));
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
  if (e) fail(CDS_ERR_CUDA, "peel: device error");
  std::vector<unsigned long long> hn(ninst), hd(ninst);
  CDS_CUDA(cudaMemcpyAsync(hn.data(), bnum.p, ninst * 8, cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaMemcpyAsync(hd.data(), bden.p, ninst * 8, cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaMemcpyAsync(out.inst_max_core.data(), imax.p, ninst * 4, cudaMemcpyDeviceToHost, s));
  uint32_t levels = 0;
  CDS_CUDA(cudaMemcpyAsync(&levels, ctl.p + CTL_LEVELS, 4, cudaMemcpyDeviceToHost, s));
  unsigned long long hph[8] = {0};
  if (c->prof) CDS_CUDA(cudaMemcpyAsync(hph, phase.p, sizeof(hph), cudaMemcpyDeviceToHost, s));
  CDS_CUDA(cudaStreamSynchronize(s));
  if (c->prof) {
    // phase breakdown of block 0 (ms) and the removal-buffer task count
    static const char *names[5] = {"peel_phase_scan", "peel_phase_collect", "peel_phase_drain",
                                   "peel_phase_barrier", "peel_tasks_x1e-6"};
    std::lock_guard<std::mutex> g(c->mu);
    for (int i = 0; i < 5; i++) {
      auto &slot = c->prof_done[names[i]];
      slot.first += 1;
      slot.second += i < 4 ? hph[i] / 1e6 : hph[i] / 1e6;
    }
  }
  out.levels = levels;
  out.max_core = 0;
  for (uint32_t i = 0; i < ninst; i++) {
    out.best_num[i] = hn[i];
    out.best_den[i] = hd[i];
    out.max_core = std::max(out.max_core, out.inst_max_core[i]);
  }
}

}  // namespace cds
