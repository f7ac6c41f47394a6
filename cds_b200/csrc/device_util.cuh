// device_util.cuh -- warp/block helpers, the bounded grid barrier and the
// device-wide exclusive scan shared by every stage.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CDS_FULL 0xFFFFFFFFu

// Error bits a device loop leaves in its status word.
enum : uint32_t {
  DEV_ERR_TIMEOUT = 1u,   // a barrier or loop ran out of its iteration budget
  DEV_ERR_OVERFLOW = 2u,  // a buffer would have overflowed; nothing was written
  DEV_ERR_INTERNAL = 4u   // an invariant check failed
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(CDS_FULL, v, o);
    if ((int)lane_id() >= o) v += t;
  }
  return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(CDS_FULL, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T t = __shfl_xor_sync(CDS_FULL, v, o);
    v = t < v ? t : v;
  }
  return v;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T t = __shfl_xor_sync(CDS_FULL, v, o);
    v = t > v ? t : v;
  }
  return v;
}

// Position of the r-th (0-based) set bit of m; m must have more than r bits.
__device__ __forceinline__ int select_bit(uint32_t m, int r) {
  int pos = 0;
  int c = __popc(m & 0xFFFFu);
  if (r >= c) { r -= c; m >>= 16; pos += 16; }
  c = __popc(m & 0xFFu);
  if (r >= c) { r -= c; m >>= 8; pos += 8; }
  c = __popc(m & 0xFu);
  if (r >= c) { r -= c; m >>= 4; pos += 4; }
  c = __popc(m & 0x3u);
  if (r >= c) { r -= c; m >>= 2; pos += 2; }
  c = (int)(m & 1u);
  if (r >= c) pos += 1;
  return pos;
}

// Warp-aggregated increment: every active lane adds 1 to base[key] with one
// atomic per distinct key in the warp and gets its own slot (the old value
// plus its rank in the group).  All 32 lanes must call it.
__device__ __forceinline__ uint32_t agg_inc(uint32_t *base, uint32_t key, bool active) {
  const uint32_t grp = __match_any_sync(CDS_FULL, active ? key : 0xFFFFFFFFu);
  uint32_t res = 0;
  if (active) {
    const int leader = __ffs(grp) - 1;
    uint32_t old = 0;
    if ((int)lane_id() == leader) old = atomicAdd(&base[key], (uint32_t)__popc(grp));
    old = __shfl_sync(grp, old, leader);
    res = old + __popc(grp & ((1u << lane_id()) - 1u));
  }
  return res;
}
// The same with 64-bit counters (a slot past 2^32).
__device__ __forceinline__ unsigned long long agg_inc_u64(unsigned long long *base, uint32_t key, bool active) {
  const uint32_t grp = __match_any_sync(CDS_FULL, active ? key : 0xFFFFFFFFu);
  unsigned long long res = 0;
  if (active) {
    const int leader = __ffs(grp) - 1;
    unsigned long long old = 0;
    if ((int)lane_id() == leader) old = atomicAdd(&base[key], (unsigned long long)__popc(grp));
    old = __shfl_sync(grp, old, leader);
    res = old + (unsigned long long)__popc(grp & ((1u << lane_id()) - 1u));
  }
  return res;
}
__device__ __forceinline__ void agg_add_u32(uint32_t *base, uint32_t key, bool active) {
  const uint32_t grp = __match_any_sync(CDS_FULL, active ? key : 0xFFFFFFFFu);
  if (active && (int)lane_id() == __ffs(grp) - 1) atomicAdd(&base[key], (uint32_t)__popc(grp));
}
__device__ __forceinline__ void agg_add_u64(unsigned long long *base, uint32_t key, bool active) {
  const uint32_t grp = __match_any_sync(CDS_FULL, active ? key : 0xFFFFFFFFu);
  if (active && (int)lane_id() == __ffs(grp) - 1) atomicAdd(&base[key], (unsigned long long)__popc(grp));
}

// base[key] += val for every active lane, where lanes in runs of the same key
// (consecutive lanes: consecutive cliques share their first members) are
// summed first and the last lane of each run adds the sum -- one atomic per
// run instead of up to 32 on one address.  Called by the whole warp.
template <typename T>
__device__ __forceinline__ void run_add(T *base, uint32_t key, T val, bool active) {
  const uint32_t lane = lane_id();
  const uint32_t kk = active ? key : 0xFFFFFFFFu;
  const uint32_t prev = __shfl_up_sync(CDS_FULL, kk, 1);
  const uint32_t heads = __ballot_sync(CDS_FULL, lane == 0 || prev != kk);
  const int start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));  // this run's first lane
  T v = active ? val : T(0);
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T o = __shfl_up_sync(CDS_FULL, v, off);
    if ((int)lane - off >= start) v += o;
  }
  const uint32_t next = __shfl_down_sync(CDS_FULL, kk, 1);
  if (active && (lane == 31 || next != kk)) atomicAdd(&base[key], v);
}

// Slot reservation with the same runs: every active lane gets a distinct
// index from base[key]++ (the run's first lane adds the run's length once
// and the others count on from it).  Called by the whole warp.
__device__ __forceinline__ uint32_t run_inc(uint32_t *base, uint32_t key, bool active) {
  const uint32_t lane = lane_id();
  const uint32_t kk = active ? key : 0xFFFFFFFFu;
  const uint32_t prev = __shfl_up_sync(CDS_FULL, kk, 1);
  const uint32_t next = __shfl_down_sync(CDS_FULL, kk, 1);
  const uint32_t heads = __ballot_sync(CDS_FULL, lane == 0 || prev != kk);
  const uint32_t tails = __ballot_sync(CDS_FULL, lane == 31 || next != kk);
  const uint32_t start = 31 - __clz(heads & (0xFFFFFFFFu >> (31 - lane)));
  const uint32_t end = __ffs(tails & (0xFFFFFFFFu << lane)) - 1;
  uint32_t old = 0;
  if (active && lane == start) old = atomicAdd(&base[key], end - start + 1);
  old = __shfl_sync(CDS_FULL, old, start);
  return old + (lane - start);
}

// 32 bytes as one 256-bit store (a whole sector, sm_100); callers pass only
// 32-byte aligned addresses.
__device__ __forceinline__ void store_sector(uint32_t *p, uint4 a, uint4 b) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(a.x), "r"(a.y), "r"(a.z),
               "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
               : "memory");
}

// Counts per key in a grid-stride loop whose keys come in long runs (the
// cliques of one network or instance are stored together): each thread keeps
// its current key's count in a register and adds it when the key changes;
// run_flush, called by the whole warp after the loop, adds what is left,
// once per warp when its lanes hold the same key.  A billion cliques of one
// key then cost a few thousand atomics instead of one per warp and step.
struct RunCount {
  uint32_t key = 0xFFFFFFFFu;
  unsigned long long n = 0;
  __device__ __forceinline__ void add(unsigned long long *base, uint32_t k, bool in) {
    if (!in) return;
    if (k != key) {
      if (n) atomicAdd(&base[key], n);
      key = k;
      n = 0;
    }
    n++;
  }
  __device__ __forceinline__ void flush(unsigned long long *base) {
    const uint32_t have = __ballot_sync(CDS_FULL, n != 0);
    if (!have) return;
    const uint32_t k0 = __shfl_sync(CDS_FULL, key, __ffs(have) - 1);
    if (__all_sync(CDS_FULL, n == 0 || key == k0)) {
      const unsigned long long t = warp_sum(n);
      if (lane_id() == 0) atomicAdd(&base[k0], t);
    } else if (n) {
      atomicAdd(&base[key], n);
    }
    n = 0;
  }
};

// 64-bit atomics on signed values through the unsigned overloads.
__device__ __forceinline__ long long atomic_add_i64(long long *p, long long v) {
  return (long long)atomicAdd((unsigned long long *)p, (unsigned long long)v);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// GPU-scope acquire load / release add (PTX memory model), cheaper than a
// full fence around a flag.
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t atom_add_release(uint32_t *p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// ---------------------------------------------------------------------------
// Grid barrier for cooperative launches.  One arrival word: block 0 adds
// 2^31 - (blocks - 1), every other block 1, so the top bit flips exactly when
// the last block arrives and the low bits return to zero -- no generation
// word and no reset, and a block that hurries on to the next barrier cannot
// flip the bit back before every block has arrived there too.  Waiters poll
// without sleeping for the first 2,048 polls (a phase is usually short),
// then with short sleeps.  Every wait is bounded: after `spin_limit` polls
// the block records DEV_ERR_TIMEOUT in *err and returns false; callers leave
// their loop when a barrier fails or *err is set.  The word must be zero at
// launch.
// ---------------------------------------------------------------------------
// Clique records of the flow networks: S = rec_slots(k) member slots (a
// power of two >= k) then S 32-bit flow words, 2S words per clique (32 bytes
// for k = 3, 4: members and flows of a clique in one sector); rec_shift(k) =
// log2(2S).
__host__ __device__ constexpr uint32_t rec_slots(uint32_t k) { return k <= 2 ? 2u : k <= 4 ? 4u : k <= 8 ? 8u : 16u; }
__host__ __device__ constexpr uint32_t rec_shift(uint32_t k) { return k <= 2 ? 2u : k <= 4 ? 3u : k <= 8 ? 4u : 5u; }

struct GridBarrier {
  unsigned int count;
  unsigned int pad[31];  // a line of its own
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, uint32_t *err,
                                          unsigned long long spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    __threadfence();  // this block's writes before its arrival
    const unsigned int old = atomicAdd(&b->count, add);
    volatile unsigned int *word = &b->count;
    int ok = 1;
    unsigned long long spins = 0;
    while (((*word ^ old) & 0x80000000u) == 0) {
      if (++spins > spin_limit) {
        atomicOr(err, DEV_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      if ((spins & 1023) == 0 && *(volatile uint32_t *)err) {  // another block gave up
        ok = 0;
        break;
      }
      if (spins > 2048) __nanosleep(256);
    }
    __threadfence();  // every block's writes before this block's reads
    if (*(volatile uint32_t *)err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// Exclusive scan of n values into out[0..n], out[n] = total (uint64).  The
// input is read through a functor so callers can scan transformed arrays.
// Host driver: scan_exclusive() in scan.cu.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *total) {
  __shared__ T s_warp[32];
  T inc = warp_inclusive_scan(v);
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane_id() == 31) s_warp[w] = inc;
  __syncthreads();
  if (w == 0) {
    T x = (int)lane_id() < nw ? s_warp[lane_id()] : T(0);
    T xi = warp_inclusive_scan(x);
    if ((int)lane_id() < nw) s_warp[lane_id()] = xi - x;
    if (lane_id() == 31) s_warp[31] = xi;  // nw <= 31 for blockDim <= 992
  }
  __syncthreads();
  T r = s_warp[w] + inc - v;
  if (total) *total = s_warp[31];
  __syncthreads();
  return r;
}
