// gen.cpp -- seeded synthetic graphs and adjacency-list text I/O (host).
//
// Randomness comes from std::mt19937_64 with uniform reals built from the raw
// 64-bit output, so a seed gives the same graph with any C++ standard library.
#include "cds_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace {

inline double u01(std::mt19937_64 &g) { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
inline uint64_t below(std::mt19937_64 &g, uint64_t n) { return n ? g() % n : 0; }

// Symmetric CSR from packed undirected keys (min << 32 | max); keys are
// sorted and de-duplicated in place.
int csr_from_keys(uint32_t n, std::vector<uint64_t> &keys, uint64_t **off_out,
                  uint32_t **adj_out) {
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  uint64_t *off = (uint64_t *)std::calloc((size_t)n + 1, sizeof(uint64_t));
  uint32_t *adj = (uint32_t *)std::malloc((2 * keys.size() + 1) * sizeof(uint32_t));
  uint64_t *cur = (uint64_t *)std::malloc(((size_t)n + 1) * sizeof(uint64_t));
  if (!off || !adj || !cur) {
    std::free(off); std::free(adj); std::free(cur);
    return -1;
  }
  for (uint64_t k : keys) { off[(k >> 32) + 1]++; off[(uint32_t)k + 1]++; }
  for (uint32_t v = 0; v < n; v++) off[v + 1] += off[v];
  std::memcpy(cur, off, ((size_t)n + 1) * sizeof(uint64_t));
  // smaller neighbours first, then larger ones: each row comes out ascending
  for (uint64_t k : keys) adj[cur[(uint32_t)k]++] = (uint32_t)(k >> 32);
  for (uint64_t k : keys) adj[cur[k >> 32]++] = (uint32_t)k;
  std::free(cur);
  *off_out = off;
  *adj_out = adj;
  return 0;
}

inline uint64_t key(uint32_t a, uint32_t b) {
  return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
}

}  // namespace

extern "C" {

void cds_free(void *p) { std::free(p); }

int cds_csr_from_edges(uint32_t n, const uint32_t *u, const uint32_t *v, uint64_t m,
                       uint64_t **off, uint32_t **adj) {
  std::vector<uint64_t> keys;
  keys.reserve(m);
  for (uint64_t i = 0; i < m; i++) {
    if (u[i] >= n || v[i] >= n) return -1;
    if (u[i] != v[i]) keys.push_back(key(u[i], v[i]));
  }
  return csr_from_keys(n, keys, off, adj);
}

int cds_gen_er(uint32_t n, double p, uint64_t seed, uint64_t **off, uint32_t **adj) {
  std::mt19937_64 g(seed);
  std::vector<uint64_t> keys;
  if (p >= 1.0) {
    for (uint32_t a = 0; a < n; a++)
      for (uint32_t b = a + 1; b < n; b++) keys.push_back(key(a, b));
  } else if (p > 0.0 && n > 1) {
    // geometric skipping over the pairs (v, w), w < v (Batagelj & Brandes 2005)
    keys.reserve((size_t)(p * 0.5 * n * (double)(n - 1) * 1.1) + 16);
    const double lq = std::log(1.0 - p);
    int64_t v = 1, w = -1;
    while (v < (int64_t)n) {
      double r = u01(g);
      w += 1 + (int64_t)std::floor(std::log(1.0 - r) / lq);
      while (w >= v && v < (int64_t)n) { w -= v; v++; }
      if (v < (int64_t)n) keys.push_back(key((uint32_t)v, (uint32_t)w));
    }
  }
  return csr_from_keys(n, keys, off, adj);
}

int cds_gen_rmat(uint32_t scale, uint32_t n, double edge_factor, double a, double b,
                 double c, uint64_t seed, uint32_t *n_out, uint64_t **off, uint32_t **adj) {
  if (scale > 31) return -1;
  const uint64_t slots = 1ull << scale;
  if (n == 0) n = (uint32_t)slots;
  if (n > slots) return -1;
  std::mt19937_64 g(seed);
  // random relabelling of the 2^scale slots, so hubs are not at small ids
  std::vector<uint32_t> perm(slots);
  for (uint64_t i = 0; i < slots; i++) perm[i] = (uint32_t)i;
  for (uint64_t i = slots - 1; i > 0; i--) std::swap(perm[i], perm[below(g, i + 1)]);
  const uint64_t samples = (uint64_t)std::llround(edge_factor * (double)slots);
  const double ab = a + b, abc = a + b + c;
  std::vector<uint64_t> keys;
  keys.reserve(samples);
  for (uint64_t e = 0; e < samples; e++) {
    for (int tries = 0; tries < 1000; tries++) {
      uint64_t x = 0, y = 0;
      for (uint32_t l = 0; l < scale; l++) {
        double r = u01(g);
        uint64_t bx = 0, by = 0;
        if (r < a) {
        } else if (r < ab) {
          by = 1;
        } else if (r < abc) {
          bx = 1;
        } else {
          bx = 1;
          by = 1;
        }
        x = (x << 1) | bx;
        y = (y << 1) | by;
      }
      uint32_t px = perm[x], py = perm[y];
      if (px >= n || py >= n) continue;
      if (px != py) keys.push_back(key(px, py));
      break;
    }
  }
  if (n_out) *n_out = n;
  return csr_from_keys(n, keys, off, adj);
}

int cds_gen_plant(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t size,
                  double p, uint64_t seed, uint64_t **off_out, uint32_t **adj_out,
                  uint32_t *members) {
  if (size > n) return -1;
  std::mt19937_64 g(seed);
  std::vector<uint32_t> pick(n);
  for (uint32_t i = 0; i < n; i++) pick[i] = i;
  for (uint32_t i = 0; i < size; i++) std::swap(pick[i], pick[i + below(g, n - i)]);
  std::vector<uint64_t> keys;
  keys.reserve(off[n] / 2 + (uint64_t)size * size / 2);
  for (uint32_t v = 0; v < n; v++)
    for (uint64_t e = off[v]; e < off[v + 1]; e++)
      if (adj[e] > v) keys.push_back(((uint64_t)v << 32) | adj[e]);
  for (uint32_t i = 0; i < size; i++)
    for (uint32_t j = i + 1; j < size; j++)
      if (u01(g) < p) keys.push_back(key(pick[i], pick[j]));
  if (members)
    for (uint32_t i = 0; i < size; i++) members[i] = pick[i];
  return csr_from_keys(n, keys, off_out, adj_out);
}

int cds_write_csr_binary(const char *path, uint32_t n, const uint64_t *off, const uint32_t *adj) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return -1;
  cds_csr_header h;
  std::memcpy(h.magic, CDS_CSR_MAGIC, 8);
  h.version = 1;
  h.reserved = 0;
  h.n = n;
  h.nnz = off[n];
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  ok = ok && std::fwrite(off, 8, (size_t)n + 1, f) == (size_t)n + 1;
  ok = ok && (h.nnz == 0 || std::fwrite(adj, 4, (size_t)h.nnz, f) == (size_t)h.nnz);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : -1;
}

int cds_read_adjlist(const char *path, uint32_t *n_out, uint64_t **off, uint32_t **adj) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return -1;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::vector<char> buf((size_t)sz + 1);
  size_t got = std::fread(buf.data(), 1, (size_t)sz, f);
  std::fclose(f);
  if (got != (size_t)sz) return -1;
  if ((size_t)sz >= sizeof(cds_csr_header) && std::memcmp(buf.data(), CDS_CSR_MAGIC, 8) == 0) {
    // the binary CSR cache: copy the arrays out, then canonicalise them like
    // any edge list (a cache written by cds_write_csr_binary already is)
    cds_csr_header h;
    std::memcpy(&h, buf.data(), sizeof(h));
    if (h.version != 1 || h.n > 0xFFFFFFFFull) return -1;
    const uint64_t need = sizeof(h) + 8 * (h.n + 1) + 4 * h.nnz;
    if ((uint64_t)sz != need) return -1;
    std::vector<uint64_t> o(h.n + 1);
    std::memcpy(o.data(), buf.data() + sizeof(h), 8 * (h.n + 1));
    if (o[0] != 0 || o[h.n] != h.nnz) return -1;
    std::vector<uint64_t> keys;
    keys.reserve(h.nnz);
    const uint32_t *a = reinterpret_cast<const uint32_t *>(buf.data() + sizeof(h) + 8 * (h.n + 1));
    for (uint64_t v = 0; v < h.n; v++) {
      if (o[v + 1] < o[v] || o[v + 1] > h.nnz) return -1;
      for (uint64_t e = o[v]; e < o[v + 1]; e++) {
        uint32_t w;
        std::memcpy(&w, a + e, 4);
        if (w >= h.n) return -1;
        if (w != v) keys.push_back(key((uint32_t)v, w));
      }
    }
    *n_out = (uint32_t)h.n;
    return csr_from_keys((uint32_t)h.n, keys, off, adj);
  }
  buf[(size_t)sz] = '\n';
  const char *p = buf.data(), *end = p + sz + 1;
  // returns 1 on a number, 0 at end of line (consumed), -1 on junk
  auto num = [&](uint64_t &x) -> int {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
    if (p >= end) return 0;
    if (*p == '\n') { p++; return 0; }
    if (*p < '0' || *p > '9') return -1;
    x = 0;
    while (p < end && *p >= '0' && *p <= '9') {
      x = x * 10 + (uint64_t)(*p++ - '0');
      if (x > 0xFFFFFFFFull) return -1;
    }
    return 1;
  };
  uint64_t n = 0, m = 0, v = 0, w = 0;
  if (num(n) != 1 || num(m) != 1) return -1;
  int r;
  while ((r = num(w)) == 1) {
  }
  if (r < 0) return -1;
  std::vector<uint64_t> keys;
  keys.reserve(m < (1ull << 32) ? m : 0);
  while (p < end) {
    r = num(v);
    if (r == 0) continue;
    if (r < 0 || v >= n) return -1;
    while ((r = num(w)) == 1) {
      if (w >= n) return -1;
      if (w != v) keys.push_back(key((uint32_t)v, (uint32_t)w));
    }
    if (r < 0) return -1;
  }
  *n_out = (uint32_t)n;
  return csr_from_keys((uint32_t)n, keys, off, adj);
}

int cds_write_adjlist(const char *path, uint32_t n, const uint64_t *off, const uint32_t *adj) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return -1;
  std::vector<char> out;
  out.reserve(1 << 20);
  char tmp[24];
  auto put = [&](uint64_t x, char sep) {
    int l = 0;
    do { tmp[l++] = (char)('0' + x % 10); x /= 10; } while (x);
    while (l) out.push_back(tmp[--l]);
    out.push_back(sep);
  };
  put(n, ' ');
  put(off[n] / 2, '\n');
  for (uint32_t v = 0; v < n; v++) {
    uint64_t b = off[v], e = off[v + 1];
    put(v, b == e ? '\n' : ' ');
    for (uint64_t i = b; i < e; i++) put(adj[i], i + 1 == e ? '\n' : ' ');
    if (out.size() > (1u << 20)) {
      std::fwrite(out.data(), 1, out.size(), f);
      out.clear();
    }
  }
  std::fwrite(out.data(), 1, out.size(), f);
  return std::fclose(f) == 0 ? 0 : -1;
}

}  // extern "C"
