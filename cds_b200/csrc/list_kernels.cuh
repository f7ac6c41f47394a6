// list_kernels.cuh -- device code of the k-clique listing (see listing.cu
// for the method).  Included by every translation unit that launches it.
#pragma once
#include "device_util.cuh"
#include "cds.h"

namespace {

constexpr int WARP_DMAX = 128;    // out-degree limit of a warp team
constexpr int BLOCK_DMAX = 1024;  // out-degree limit for rows in shared memory
constexpr int DFS_WMAX = 32;      // bitmap words a DFS mask may need (k >= 5)

struct ListParams {
  const uint64_t *doff;
  const uint32_t *dadj;
  const uint32_t *outdeg;
  const uint32_t *roots;
  const uint32_t *nroots;          // root count, on the device
  uint32_t *work;                  // dynamic scheduling cursor
  uint32_t *cdeg;                  // pass 1: clique degree (atomic), when cdeg64 is null
  unsigned long long *cdeg64;      // pass 1: clique degree as u64 (no 2^32 cap)
  unsigned long long *root_cnt;    // pass 1: cliques per root vertex
  const unsigned long long *base;  // pass 2: first clique index per vertex
  uint32_t *out;                   // pass 2: clique records
  uint32_t dmax;                   // team capacity (entries)
  uint32_t team_words;             // shared-memory words per team
  uint32_t *rows_global;           // block teams: rows outside shared memory
  uint64_t rows_slab;              // words per block slab
  uint32_t *err;
  uint32_t k;                      // clique size (used by the generic k >= 5 path)
};

template <bool TB>
struct Team {
  __device__ __forceinline__ static int size() { return TB ? (int)blockDim.x : 32; }
  __device__ __forceinline__ static int rank() { return TB ? (int)threadIdx.x : (int)lane_id(); }
  __device__ __forceinline__ static int warps() { return TB ? (int)(blockDim.x >> 5) : 1; }
  __device__ __forceinline__ static int warp() { return TB ? (int)(threadIdx.x >> 5) : 0; }
  __device__ __forceinline__ static void sync() {
    if (TB) __syncthreads();
    else __syncwarp();
  }
  // exclusive scan of one value per team thread; *tot = team total
  template <class T>
  __device__ __forceinline__ static T scan(T v, T *tot) {
    if (TB) return block_exclusive_scan<T>(v, tot);
    T inc = warp_inclusive_scan(v);
    *tot = __shfl_sync(CDS_FULL, inc, 31);
    return inc - v;
  }
  template <class T>
  __device__ __forceinline__ static T sum(T v) {
    T tot;
    scan<T>(v, &tot);
    return tot;
  }
};

// first index i with P[i+1] > p, for P ascending with P[0] = 0
__device__ __forceinline__ uint32_t find_row(const uint32_t *P, uint32_t d, uint32_t p) {
  uint32_t lo = 0, hi = d;  // answer in [0, d)
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (P[mid] <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t nth_in_row(const uint32_t *row, uint32_t r) {
  for (uint32_t w = 0;; w++) {
    const uint32_t c = __popc(row[w]);
    if (r < c) return (w << 5) + (uint32_t)select_bit(row[w], (int)r);
    r -= c;
  }
}

// Enumerates the (depth)-cliques inside mask M (W words) with DFS over the
// bitmap rows; calls leaf(path, depth) for each.  Only used for k >= 5.
template <class Leaf>
__device__ void dfs_cliques(const uint32_t *rows, uint32_t rs, uint32_t W, const uint32_t *M,
                            int depth, Leaf leaf) {
  uint32_t stack[CDS_MAX_K][DFS_WMAX];
  uint32_t path[CDS_MAX_K];
  uint32_t pos[CDS_MAX_K];
  for (uint32_t w = 0; w < W; w++) stack[0][w] = M[w];
  int lvl = 0;
  pos[0] = 0;
  while (lvl >= 0) {
    // next set bit of stack[lvl] at or after pos[lvl]
    uint32_t b = pos[lvl];
    uint32_t found = 0xFFFFFFFFu;
    while ((b >> 5) < W) {
      const uint32_t word = stack[lvl][b >> 5] & (0xFFFFFFFFu << (b & 31));
      if (word) { found = ((b >> 5) << 5) + (uint32_t)(__ffs(word) - 1); break; }
      b = ((b >> 5) + 1) << 5;
    }
    if (found == 0xFFFFFFFFu) { lvl--; continue; }
    pos[lvl] = found + 1;
    path[lvl] = found;
    if (lvl + 1 == depth) {
      leaf(path, depth);
      continue;
    }
    const uint32_t *row = rows + found * rs;
    uint32_t any = 0;
    for (uint32_t w = 0; w < W; w++) {
      stack[lvl + 1][w] = stack[lvl][w] & row[w];
      any |= stack[lvl + 1][w];
    }
    if (any) {
      lvl++;
      pos[lvl] = 0;
    }
  }
}

// K = 3 and K = 4 are specialised; K = 0 is the generic path for k >= 5.
template <int K, bool WRITE, bool TB>
__global__ void k_list(ListParams p) {
  using T = Team<TB>;
  const int KK = K ? K : (int)p.k;
  extern __shared__ uint32_t sm[];
  __shared__ uint32_t s_root;
  uint32_t *S = sm + (TB ? 0u : (threadIdx.x >> 5) * p.team_words);
  uint32_t *A = S;                  // [dmax]
  uint32_t *P = A + p.dmax;         // [dmax+1] row-popcount prefix
  uint32_t *cnt = P + p.dmax + 1;   // [dmax] local clique degrees
  uint32_t *rows = (TB && p.rows_global) ? p.rows_global + (uint64_t)blockIdx.x * p.rows_slab
                                         : cnt + p.dmax;
  const int tr = T::rank(), ts = T::size();
  const uint32_t nroots = *p.nroots;
  for (;;) {
    uint32_t r;
    if (TB) {
      if (threadIdx.x == 0) s_root = atomicAdd(p.work, 1u);
      __syncthreads();
      r = s_root;
      __syncthreads();
    } else {
      if (lane_id() == 0) r = atomicAdd(p.work, 1u);
      r = __shfl_sync(CDS_FULL, r, 0);
    }
    if (r >= nroots) break;
    const uint32_t u = p.roots[r];
    const uint32_t d = p.outdeg[u];
    if (d > p.dmax) {  // classification guarantees d <= dmax
      if (tr == 0) atomicOr(p.err, DEV_ERR_INTERNAL);
      continue;
    }
    const uint32_t W = (d + 31) >> 5;
    if (K == 0 && W > (uint32_t)DFS_WMAX) {  // DFS masks are limited to DFS_WMAX words
      if (tr == 0) atomicOr(p.err, DEV_ERR_OVERFLOW);
      continue;
    }
    const uint32_t rs = W | 1u;  // odd stride: lanes reading different rows hit different banks
    const uint32_t *Au = p.dadj + p.doff[u];
    for (uint32_t i = (uint32_t)tr * 4; i < d; i += (uint32_t)ts * 4) {
      const uint4 q = *reinterpret_cast<const uint4 *>(Au + i);
      A[i] = q.x;
      if (i + 1 < d) A[i + 1] = q.y;
      if (i + 2 < d) A[i + 2] = q.z;
      if (i + 3 < d) A[i + 3] = q.w;
    }
    for (uint32_t i = tr; i < d * rs; i += ts) rows[i] = 0;
    T::sync();
    // local adjacency bitmap
    for (uint32_t i = T::warp(); i < d; i += T::warps()) {
      const uint32_t a = A[i];
      const uint32_t da = p.outdeg[a];
      const uint32_t *Aa = p.dadj + p.doff[a];
      uint32_t *row = rows + i * rs;
      const uint32_t lo_id = A[0], hi_id = A[d - 1];
      for (uint32_t t = lane_id(); t < da; t += 32) {
        const uint32_t b = Aa[t];
        if (b < lo_id || b > hi_id) continue;
        uint32_t lo = 0, hi = d;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (A[mid] < b) lo = mid + 1;
          else hi = mid;
        }
        if (lo < d && A[lo] == b) atomicOr(&row[lo >> 5], 1u << (lo & 31));
      }
    }
    T::sync();
    // P = exclusive prefix of row popcounts; cnt[i] = popcount (pass 1, k = 3)
    uint32_t carry = 0;
    for (uint32_t i0 = 0; i0 < d; i0 += ts) {
      const uint32_t i = i0 + tr;
      uint32_t v = 0;
      if (i < d)
        for (uint32_t w = 0; w < W; w++) v += __popc(rows[i * rs + w]);
      uint32_t tot;
      const uint32_t ex = T::template scan<uint32_t>(v, &tot);
      if (i < d) {
        P[i] = carry + ex;
        if (!WRITE) cnt[i] = (K == 3) ? v : 0u;
      }
      carry += tot;
    }
    if (tr == 0) P[d] = carry;
    T::sync();
    const uint32_t npairs = carry;
    unsigned long long mine = 0;  // cliques counted by this thread
    if (K == 3) {
      if (!WRITE) {
        for (uint32_t q = tr; q < npairs; q += ts) {
          const uint32_t i = find_row(P, d, q);
          const uint32_t j = nth_in_row(rows + i * rs, q - P[i]);
          atomicAdd(&cnt[j], 1u);
        }
        mine = (tr == 0) ? npairs : 0;
      } else {
        const unsigned long long b0 = p.base[u];
        for (uint32_t q = tr; q < npairs; q += ts) {
          const uint32_t i = find_row(P, d, q);
          const uint32_t j = nth_in_row(rows + i * rs, q - P[i]);
          uint32_t *o = p.out + (b0 + q) * 3;
          o[0] = u;
          o[1] = A[i];
          o[2] = A[j];
        }
      }
    } else {
      unsigned long long wcarry = WRITE ? p.base[u] : 0ull;
      for (uint32_t q0 = 0; q0 < npairs; q0 += ts) {
        const uint32_t q = q0 + tr;
        uint32_t i = 0, j = 0;
        unsigned long long c = 0;
        uint32_t M[K == 4 ? 4 : DFS_WMAX];
        const bool small = (K == 4) && W <= 4;
        if (q < npairs) {
          i = find_row(P, d, q);
          j = nth_in_row(rows + i * rs, q - P[i]);
          const uint32_t *ri = rows + i * rs, *rj = rows + j * rs;
          if (K == 4) {
            if (small) {
              for (uint32_t w = 0; w < W; w++) {
                M[w] = ri[w] & rj[w];
                c += __popc(M[w]);
              }
            } else {
              for (uint32_t w = 0; w < W; w++) c += __popc(ri[w] & rj[w]);
            }
          } else {
            uint32_t any = 0;
            for (uint32_t w = 0; w < W; w++) {
              M[w] = ri[w] & rj[w];
              any |= M[w];
            }
            if (any)
              dfs_cliques(rows, rs, W, M, KK - 3,
                          [&](const uint32_t *, int) { c++; });
          }
        }
        if (!WRITE) {
          if (c) {
            mine += c;
            atomicAdd(&cnt[i], (uint32_t)c);
            atomicAdd(&cnt[j], (uint32_t)c);
            const uint32_t *ri = rows + i * rs, *rj = rows + j * rs;
            if (K == 4) {
              for (uint32_t w = 0; w < W; w++) {
                uint32_t m = ri[w] & rj[w];
                while (m) {
                  atomicAdd(&cnt[(w << 5) + (uint32_t)(__ffs(m) - 1)], 1u);
                  m &= m - 1;
                }
              }
            } else {
              dfs_cliques(rows, rs, W, M, KK - 3, [&](const uint32_t *path, int depth) {
                for (int t = 0; t < depth; t++) atomicAdd(&cnt[path[t]], 1u);
              });
            }
          }
        } else {
          unsigned long long tot;
          const unsigned long long ex = T::template scan<unsigned long long>(c, &tot);
          if (c) {
            unsigned long long o = wcarry + ex;
            const uint32_t ai = A[i], aj = A[j];
            if (K == 4) {
              // a record that starts a 32-byte sector waits for its successor,
              // and the two go out as one 32-byte store (a whole sector)
              // instead of two half-sector stores
              const uint32_t *ri = rows + i * rs, *rj = rows + j * rs;
              uint4 pend = make_uint4(0u, 0u, 0u, 0u);
              bool has = false;
              for (uint32_t w = 0; w < W; w++) {
                uint32_t m = small ? M[w] : (ri[w] & rj[w]);
                while (m) {
                  const uint32_t l = (w << 5) + (uint32_t)(__ffs(m) - 1);
                  m &= m - 1;
                  const uint4 r = make_uint4(u, ai, aj, A[l]);
                  if (has) {
                    store_sector(p.out + (o - 1) * 4, pend, r);
                    has = false;
                  } else if ((reinterpret_cast<uintptr_t>(p.out + o * 4) & 31u) == 0) {
                    pend = r;
                    has = true;
                  } else {
                    *reinterpret_cast<uint4 *>(p.out + o * 4) = r;
                  }
                  o++;
                }
              }
              if (has) *reinterpret_cast<uint4 *>(p.out + (o - 1) * 4) = pend;
            } else {
              dfs_cliques(rows, rs, W, M, KK - 3, [&](const uint32_t *path, int depth) {
                uint32_t *rec = p.out + o * (unsigned long long)KK;
                rec[0] = u;
                rec[1] = ai;
                rec[2] = aj;
                for (int t = 0; t < depth; t++) rec[3 + t] = A[path[t]];
                o++;
              });
            }
          }
          wcarry += tot;
        }
      }
    }
    if (!WRITE) {
      T::sync();
      for (uint32_t i = tr; i < d; i += ts)
        if (cnt[i]) {
          if (p.cdeg64) atomicAdd(&p.cdeg64[A[i]], (unsigned long long)cnt[i]);
          else atomicAdd(&p.cdeg[A[i]], cnt[i]);
        }
      const unsigned long long total = T::template sum<unsigned long long>(mine);
      if (tr == 0) {
        p.root_cnt[u] = total;
        if (total) {
          if (p.cdeg64) atomicAdd(&p.cdeg64[u], total);
          else atomicAdd(&p.cdeg[u], (uint32_t)total);
        }
      }
    }
    T::sync();
  }
}

// roots with out-degree >= k-1, split by team size
__global__ void k_classify(const uint32_t *__restrict__ outdeg, uint32_t n, uint32_t kmin,
                           uint32_t warp_dmax, uint32_t *wl, uint32_t *wn, uint32_t *bl,
                           uint32_t *bn) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t d = outdeg[v];
    if (d < kmin) continue;
    if (d <= warp_dmax) wl[atomicAdd(wn, 1u)] = v;
    else bl[atomicAdd(bn, 1u)] = v;
  }
}

}  // namespace
