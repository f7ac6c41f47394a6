/* cds_oracle.c -- CPU restatement of the reference k-clique densest-subgraph
 * pipeline (wajidmanzoor/CDS, cpuCode/c++/src/helpers.cpp, CDS::DSD at
 * :1422-1589).  TEST INFRASTRUCTURE ONLY: the checker used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The product never
 * links, loads or calls it.
 *
 * Pinning: tests/test_oracle.py checks this file against the reference
 * program compiled from its own sources (oracle/_ref) through golden vectors
 * in tests/golden/ -- clique counts, clique degrees, the full peel table and
 * the final density -- and against brute force on small graphs.
 *
 * Where this restatement departs from the reference, on purpose:
 *  - Arithmetic is exact.  The reference keeps capacities in float and stops
 *    its binary search at a gap of max(1/(n(n-1)), 0.01) (helpers.cpp:1259-
 *    1286), so it can return a set slightly below the optimum.  Here the
 *    density guess is a fraction p/q, capacities are scaled by q into int64,
 *    and the search ends with a max-flow certificate at alpha = rho*.
 *  - The answer inside a component is the maximal densest set (the vertex
 *    part of the maximal min-cut source side at alpha = rho*), which is unique;
 *    the reference returns the minimal source side at its last failing alpha.
 *    Both have the optimal density; they differ only on ties.
 *  - The UB2 bound (helpers.cpp:1186-1198) is not used: it is not an upper
 *    bound in general.  No bound is used to skip work at all.
 *  - Peel selection picks the minimum current clique degree with ties to the
 *    lowest id, as helpers.cpp:92-100 intends; the reference starts that scan
 *    at 0xFFFFFF, which differs only when every remaining degree is >= 2^24-1.
 *  - Counts are int64 (the reference peel counts in int, helpers.cpp:38).
 *  - A graph with no k-clique returns density 0 and an empty set.
 */
#include "cds_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void oracle_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* growable arrays                                                           */
/* ------------------------------------------------------------------------ */
typedef struct { uint32_t *a; uint64_t n, cap; } vec32;
typedef struct { uint64_t *a; uint64_t n, cap; } vec64;

static int v32_push(vec32 *v, uint32_t x) {
  if (v->n == v->cap) {
    uint64_t c = v->cap ? v->cap * 2 : 1024;
    uint32_t *p = (uint32_t *)realloc(v->a, c * sizeof(uint32_t));
    if (!p) return -1;
    v->a = p; v->cap = c;
  }
  v->a[v->n++] = x;
  return 0;
}
static int v64_push(vec64 *v, uint64_t x) {
  if (v->n == v->cap) {
    uint64_t c = v->cap ? v->cap * 2 : 1024;
    uint64_t *p = (uint64_t *)realloc(v->a, c * sizeof(uint64_t));
    if (!p) return -1;
    v->a = p; v->cap = c;
  }
  v->a[v->n++] = x;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* reader: cpuCode/c++/src/graph.cpp:9-52                                    */
/* ------------------------------------------------------------------------ */
static int next_int(const char **pp, const char *end, long long *out, int stop_at_nl) {
  const char *p = *pp;
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || (!stop_at_nl && *p == '\n'))) p++;
  if (p >= end || *p == '\n') { *pp = p; return 0; }
  int neg = 0;
  if (*p == '-') { neg = 1; p++; }
  if (p >= end || *p < '0' || *p > '9') { *pp = p; return -1; }
  long long x = 0;
  while (p < end && *p >= '0' && *p <= '9') x = x * 10 + (*p++ - '0');
  *out = neg ? -x : x;
  *pp = p;
  return 1;
}

int oracle_read_adjlist(const char *path, uint32_t *n_out, uint64_t **off_out,
                        uint32_t **adj_out) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *buf = (char *)malloc((size_t)sz + 1);
  if (!buf || fread(buf, 1, (size_t)sz, f) != (size_t)sz) { fclose(f); free(buf); return -1; }
  fclose(f);
  buf[sz] = 0;
  const char *p = buf, *end = buf + sz;
  long long n = 0, m = 0;
  if (next_int(&p, end, &n, 1) != 1 || next_int(&p, end, &m, 1) != 1 || n < 0) { free(buf); return -1; }
  vec64 pairs = {0};  /* (v << 32) | nbr in file order */
  while (p < end) {
    while (p < end && *p != '\n') p++;  /* rest of the previous line */
    if (p < end) p++;
    long long v;
    int r = next_int(&p, end, &v, 1);
    if (r == 0) continue;
    if (r < 0 || v < 0 || v >= n) { free(buf); free(pairs.a); return -1; }
    long long w;
    while ((r = next_int(&p, end, &w, 1)) == 1) {
      if (w < 0 || w >= n) { free(buf); free(pairs.a); return -1; }
      if (w == v) continue;  /* graph.cpp:29-30 drops self-loops */
      if (v64_push(&pairs, ((uint64_t)v << 32) | (uint64_t)w)) { free(buf); free(pairs.a); return -1; }
    }
    if (r < 0) { free(buf); free(pairs.a); return -1; }
  }
  free(buf);
  uint64_t *off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  uint32_t *adj = (uint32_t *)malloc((pairs.n ? pairs.n : 1) * sizeof(uint32_t));
  if (!off || !adj) { free(off); free(adj); free(pairs.a); return -1; }
  for (uint64_t i = 0; i < pairs.n; i++) off[(pairs.a[i] >> 32) + 1]++;
  for (long long i = 0; i < n; i++) off[i + 1] += off[i];
  uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  if (!cur) { free(off); free(adj); free(pairs.a); return -1; }
  memcpy(cur, off, ((size_t)n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < pairs.n; i++) adj[cur[pairs.a[i] >> 32]++] = (uint32_t)pairs.a[i];
  free(cur);
  free(pairs.a);
  *n_out = (uint32_t)n;
  *off_out = off;
  *adj_out = adj;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* degeneracy order and DAG: helpers.cpp:248-315 (bin-sort core peel) and    */
/* helpers.cpp:349-371 (orientation).  The reference orients each edge       */
/* toward the vertex peeled earlier; this file orients it toward the vertex  */
/* peeled later, which bounds out-degrees by the degeneracy.  The set of     */
/* k-cliques does not depend on the orientation.                              */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint32_t n;
  uint64_t *off;
  uint32_t *adj;  /* out-neighbours, ascending id */
  uint32_t maxout;
} dag_t;

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

static int build_dag(uint32_t n, const uint64_t *off, const uint32_t *adj, dag_t *d) {
  uint32_t *deg = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
  uint32_t *pos = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
  uint32_t *vert = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
  uint32_t *rank = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
  uint32_t maxd = 0;
  if (!deg || !pos || !vert || !rank) goto fail;
  for (uint32_t v = 0; v < n; v++) {
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
    if (deg[v] > maxd) maxd = deg[v];
  }
  uint32_t *bin = (uint32_t *)calloc((size_t)maxd + 2, sizeof(uint32_t));
  if (!bin) goto fail;
  for (uint32_t v = 0; v < n; v++) bin[deg[v]]++;
  uint32_t start = 0;
  for (uint32_t d0 = 0; d0 <= maxd; d0++) { uint32_t c = bin[d0]; bin[d0] = start; start += c; }
  for (uint32_t v = 0; v < n; v++) { pos[v] = bin[deg[v]]; vert[pos[v]] = v; bin[deg[v]]++; }
  for (uint32_t d0 = maxd; d0 > 0; d0--) bin[d0] = bin[d0 - 1];
  bin[0] = 0;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t v = vert[i];
    rank[v] = i;
    for (uint64_t e = off[v]; e < off[v + 1]; e++) {
      uint32_t u = adj[e];
      if (deg[u] > deg[v]) {
        uint32_t du = deg[u], pu = pos[u], pw = bin[du], w = vert[pw];
        if (u != w) { pos[u] = pw; vert[pu] = w; pos[w] = pu; vert[pw] = u; }
        bin[du]++;
        deg[u]--;
      }
    }
  }
  free(bin);
  d->n = n;
  d->off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  if (!d->off) goto fail;
  for (uint32_t v = 0; v < n; v++) {
    uint64_t c = 0;
    for (uint64_t e = off[v]; e < off[v + 1]; e++) c += rank[adj[e]] > rank[v];
    d->off[v + 1] = d->off[v] + c;
  }
  d->adj = (uint32_t *)malloc((d->off[n] ? d->off[n] : 1) * sizeof(uint32_t));
  if (!d->adj) goto fail;
  d->maxout = 0;
  for (uint32_t v = 0; v < n; v++) {
    uint64_t w = d->off[v];
    for (uint64_t e = off[v]; e < off[v + 1]; e++)
      if (rank[adj[e]] > rank[v]) d->adj[w++] = adj[e];
    uint64_t len = d->off[v + 1] - d->off[v];
    qsort(d->adj + d->off[v], (size_t)len, sizeof(uint32_t), cmp_u32);
    if (len > d->maxout) d->maxout = (uint32_t)len;
  }
  free(deg); free(pos); free(vert); free(rank);
  return 0;
fail:
  free(deg); free(pos); free(vert); free(rank);
  return -1;
}

static void free_dag(dag_t *d) { free(d->off); free(d->adj); }

/* ------------------------------------------------------------------------ */
/* k-clique enumeration: helpers.cpp:373-511 (listCliques).  The reference  */
/* narrows the candidate set level by level with labels; this file narrows  */
/* it by intersecting sorted out-lists.  Each clique is produced once, in   */
/* orientation order.                                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  const dag_t *d;
  uint32_t k;
  uint32_t clique[64];
  uint32_t **buf;   /* buf[level] holds the candidates of that level */
  /* sink */
  int64_t total;
  int64_t *degree;        /* optional per-vertex counts */
  vec32 *store;           /* optional materialised cliques */
  const uint8_t *in_set;  /* optional filter: count only cliques inside */
  int err;
} enum_t;

static void emit(enum_t *e) {
  if (e->in_set) {
    for (uint32_t i = 0; i < e->k; i++)
      if (!e->in_set[e->clique[i]]) return;
  }
  e->total++;
  if (e->degree)
    for (uint32_t i = 0; i < e->k; i++) e->degree[e->clique[i]]++;
  if (e->store)
    for (uint32_t i = 0; i < e->k; i++)
      if (v32_push(e->store, e->clique[i])) e->err = 1;
}

static void enum_rec(enum_t *e, uint32_t level, const uint32_t *cand, uint32_t len) {
  if (level == e->k - 1) {
    for (uint32_t i = 0; i < len; i++) { e->clique[level] = cand[i]; emit(e); }
    return;
  }
  uint32_t *next = e->buf[level + 1];
  for (uint32_t i = 0; i < len; i++) {
    uint32_t c = cand[i];
    e->clique[level] = c;
    const uint32_t *o = e->d->adj + e->d->off[c];
    uint32_t olen = (uint32_t)(e->d->off[c + 1] - e->d->off[c]);
    uint32_t a = 0, b = 0, m = 0;
    while (a < len && b < olen) {
      if (cand[a] < o[b]) a++;
      else if (cand[a] > o[b]) b++;
      else { next[m++] = cand[a]; a++; b++; }
    }
    if (m >= e->k - 1 - level) enum_rec(e, level + 1, next, m);
  }
}

static int enumerate_roots(const dag_t *d, uint32_t k, enum_t *e, uint32_t stride, uint32_t phase);

static int enumerate(const dag_t *d, uint32_t k, enum_t *e) { return enumerate_roots(d, k, e, 1, 0); }

/* Roots u with u % stride == phase only (stride 1: every clique). */
static int enumerate_roots(const dag_t *d, uint32_t k, enum_t *e, uint32_t stride, uint32_t phase) {
  if (k < 2 || k > 64 || stride == 0) return -1;
  e->d = d;
  e->k = k;
  e->buf = (uint32_t **)calloc(k + 1, sizeof(uint32_t *));
  if (!e->buf) return -1;
  for (uint32_t l = 0; l <= k; l++) {
    e->buf[l] = (uint32_t *)malloc(((size_t)d->maxout + 1) * sizeof(uint32_t));
    if (!e->buf[l]) return -1;
  }
  for (uint32_t u = phase; u < d->n; u += stride) {
    e->clique[0] = u;
    uint32_t len = (uint32_t)(d->off[u + 1] - d->off[u]);
    if (len >= k - 1) enum_rec(e, 1, d->adj + d->off[u], len);
  }
  for (uint32_t l = 0; l <= k; l++) free(e->buf[l]);
  free(e->buf);
  return e->err ? -1 : 0;
}

int64_t oracle_count_cliques(uint32_t n, const uint64_t *off, const uint32_t *adj,
                             uint32_t k, int64_t *clique_degree) {
  dag_t d;
  if (build_dag(n, off, adj, &d)) return -1;
  enum_t e;
  memset(&e, 0, sizeof(e));
  if (clique_degree) memset(clique_degree, 0, (size_t)n * sizeof(int64_t));
  e.degree = clique_degree;
  int r = enumerate(&d, k, &e);
  free_dag(&d);
  return r ? -1 : e.total;
}

int64_t oracle_count_cliques_sampled(uint32_t n, const uint64_t *off, const uint32_t *adj,
                                     uint32_t k, uint32_t stride, uint32_t phase) {
  dag_t d;
  if (build_dag(n, off, adj, &d)) return -1;
  enum_t e;
  memset(&e, 0, sizeof(e));
  int r = enumerate_roots(&d, k, &e, stride, phase);
  free_dag(&d);
  return r ? -1 : e.total;
}

int64_t oracle_count_in_set(uint32_t n, const uint64_t *off, const uint32_t *adj,
                            uint32_t k, const uint8_t *in_set) {
  dag_t d;
  if (build_dag(n, off, adj, &d)) return -1;
  enum_t e;
  memset(&e, 0, sizeof(e));
  e.in_set = in_set;
  int r = enumerate(&d, k, &e);
  free_dag(&d);
  return r ? -1 : e.total;
}

/* ------------------------------------------------------------------------ */
/* clique-core peel: helpers.cpp:16-150.  The reference picks the next      */
/* vertex by a linear scan for the minimum current clique degree (lowest id  */
/* on ties, :92-100) and re-lists the cliques of its neighbourhood          */
/* (:111, :152-228) to subtract them.  Here a binary heap ordered by        */
/* (degree, id) makes the same choice and a vertex->clique incidence list   */
/* makes the same subtraction.                                               */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t *deg;
  uint32_t *heap;
  int64_t *hpos;
  uint32_t size;
} heap_t;

static int h_less(const heap_t *h, uint32_t a, uint32_t b) {
  return h->deg[a] < h->deg[b] || (h->deg[a] == h->deg[b] && a < b);
}
static void h_swap(heap_t *h, uint32_t i, uint32_t j) {
  uint32_t a = h->heap[i], b = h->heap[j];
  h->heap[i] = b; h->heap[j] = a;
  h->hpos[b] = i; h->hpos[a] = j;
}
static void h_up(heap_t *h, uint32_t i) {
  while (i > 0) {
    uint32_t p = (i - 1) / 2;
    if (!h_less(h, h->heap[i], h->heap[p])) break;
    h_swap(h, i, p);
    i = p;
  }
}
static void h_down(heap_t *h, uint32_t i) {
  for (;;) {
    uint32_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < h->size && h_less(h, h->heap[l], h->heap[m])) m = l;
    if (r < h->size && h_less(h, h->heap[r], h->heap[m])) m = r;
    if (m == i) break;
    h_swap(h, i, m);
    i = m;
  }
}

typedef struct {
  uint32_t n, k;
  int64_t m;          /* |Psi| */
  uint32_t *cl;       /* m*k members */
  uint32_t *order;    /* removal order */
  int64_t *rdeg;      /* clique degree at removal */
  int64_t *left;      /* cliques left after removal */
  int64_t *core;      /* clique-core number */
} peel_t;

static void free_peel(peel_t *p) {
  free(p->cl); free(p->order); free(p->rdeg); free(p->left); free(p->core);
}

static int run_peel(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t k,
                    peel_t *P) {
  memset(P, 0, sizeof(*P));
  P->n = n;
  P->k = k;
  dag_t d;
  if (build_dag(n, off, adj, &d)) return -1;
  vec32 store = {0};
  enum_t e;
  memset(&e, 0, sizeof(e));
  e.store = &store;
  int r = enumerate(&d, k, &e);
  free_dag(&d);
  if (r) { free(store.a); return -1; }
  P->m = e.total;
  P->cl = store.a;
  int64_t m = P->m;
  P->order = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  P->rdeg = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  P->left = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  P->core = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  uint64_t *ioff = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  uint64_t *icur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  uint32_t *inc = (uint32_t *)malloc(((size_t)m * k + 1) * sizeof(uint32_t));
  uint8_t *dead = (uint8_t *)calloc((size_t)m + 1, 1);
  heap_t h;
  h.deg = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  h.heap = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  h.hpos = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  if (!P->order || !P->rdeg || !P->left || !P->core || !ioff || !icur || !inc || !dead ||
      !h.deg || !h.heap || !h.hpos) {
    free(ioff); free(icur); free(inc); free(dead); free(h.deg); free(h.heap); free(h.hpos);
    free_peel(P);
    return -1;
  }
  for (int64_t c = 0; c < m; c++)
    for (uint32_t j = 0; j < k; j++) { ioff[P->cl[c * k + j] + 1]++; h.deg[P->cl[c * k + j]]++; }
  for (uint32_t v = 0; v < n; v++) ioff[v + 1] += ioff[v];
  memcpy(icur, ioff, ((size_t)n + 1) * sizeof(uint64_t));
  for (int64_t c = 0; c < m; c++)
    for (uint32_t j = 0; j < k; j++) inc[icur[P->cl[c * k + j]]++] = (uint32_t)c;
  h.size = n;
  for (uint32_t v = 0; v < n; v++) { h.heap[v] = v; h.hpos[v] = v; }
  for (int64_t i = (int64_t)n / 2; i >= 0; i--) h_down(&h, (uint32_t)i);
  int64_t alive = m, run = 0;
  for (uint32_t step = 0; step < n; step++) {
    uint32_t v = h.heap[0];
    h.size--;
    if (h.size) { h_swap(&h, 0, h.size); h_down(&h, 0); }
    h.hpos[v] = -1;
    int64_t rd = h.deg[v];
    for (uint64_t t = ioff[v]; t < ioff[v + 1]; t++) {
      uint32_t c = inc[t];
      if (dead[c]) continue;
      dead[c] = 1;
      alive--;
      for (uint32_t j = 0; j < k; j++) {
        uint32_t w = P->cl[(int64_t)c * k + j];
        if (w == v) continue;
        h.deg[w]--;
        if (h.hpos[w] >= 0) h_up(&h, (uint32_t)h.hpos[w]);
      }
    }
    h.deg[v] = 0;
    if (rd > run) run = rd;
    P->order[step] = v;
    P->rdeg[step] = rd;
    P->left[step] = alive;
    P->core[v] = run;
  }
  free(ioff); free(icur); free(inc); free(dead); free(h.deg); free(h.heap); free(h.hpos);
  return 0;
}

int64_t oracle_peel(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t k,
                    uint32_t *order, int64_t *removal_degree, int64_t *cliques_left,
                    int64_t *core) {
  peel_t P;
  if (run_peel(n, off, adj, k, &P)) return -1;
  if (order) memcpy(order, P.order, (size_t)n * sizeof(uint32_t));
  if (removal_degree) memcpy(removal_degree, P.rdeg, (size_t)n * sizeof(int64_t));
  if (cliques_left) memcpy(cliques_left, P.left, (size_t)n * sizeof(int64_t));
  if (core) memcpy(core, P.core, (size_t)n * sizeof(int64_t));
  int64_t m = P.m;
  free_peel(&P);
  return m;
}

/* ------------------------------------------------------------------------ */
/* max-flow on the reference's clique-vertex network (helpers.cpp:1302-1341) */
/* at alpha = p/q, every capacity multiplied by q:                           */
/*   s->v  q*deg(v)    v->t  k*p    v->psi  q    psi->v  q*(k-1)            */
/* solved by Dinic (the reference uses Edmonds-Karp, :1343-1405).           */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint32_t N;                 /* nodes */
  uint64_t A;                 /* arcs */
  uint32_t *to;
  int64_t *cap;
  uint64_t *head;             /* CSR over arcs: head[N+1] */
  uint64_t *arcs;             /* arc ids grouped by tail */
} net_t;

static void free_net(net_t *g) { free(g->to); free(g->cap); free(g->head); free(g->arcs); }

/* nodes: vertices [0,nc), cliques [nc,nc+mc), s = nc+mc, t = s+1 */
static int build_net(net_t *g, uint32_t nc, int64_t mc, uint32_t k, const uint32_t *cm,
                     const int64_t *deg, int64_t p, int64_t q) {
  g->N = nc + (uint32_t)mc + 2;
  uint32_t s = nc + (uint32_t)mc, t = s + 1;
  g->A = 2 * (2 * (uint64_t)mc * k + 2 * (uint64_t)nc);
  g->to = (uint32_t *)malloc(g->A * sizeof(uint32_t));
  g->cap = (int64_t *)malloc(g->A * sizeof(int64_t));
  uint32_t *tail = (uint32_t *)malloc(g->A * sizeof(uint32_t));
  g->head = (uint64_t *)calloc((size_t)g->N + 1, sizeof(uint64_t));
  g->arcs = (uint64_t *)malloc(g->A * sizeof(uint64_t));
  if (!g->to || !g->cap || !tail || !g->head || !g->arcs) { free(tail); return -1; }
  uint64_t a = 0;
#define ADD(u, v, c)                                   \
  do {                                                 \
    tail[a] = (u); g->to[a] = (v); g->cap[a] = (c); a++; \
    tail[a] = (v); g->to[a] = (u); g->cap[a] = 0; a++;   \
  } while (0)
  for (int64_t c = 0; c < mc; c++)
    for (uint32_t j = 0; j < k; j++) {
      uint32_t v = cm[c * k + j];
      ADD(nc + (uint32_t)c, v, q * (int64_t)(k - 1));
      ADD(v, nc + (uint32_t)c, q);
    }
  for (uint32_t v = 0; v < nc; v++) {
    ADD(s, v, q * deg[v]);
    ADD(v, t, (int64_t)k * p);
  }
#undef ADD
  for (uint64_t i = 0; i < a; i++) g->head[tail[i] + 1]++;
  for (uint32_t u = 0; u < g->N; u++) g->head[u + 1] += g->head[u];
  uint64_t *cur = (uint64_t *)malloc(((size_t)g->N + 1) * sizeof(uint64_t));
  if (!cur) { free(tail); return -1; }
  memcpy(cur, g->head, ((size_t)g->N + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < a; i++) g->arcs[cur[tail[i]]++] = i;
  free(cur);
  free(tail);
  return 0;
}

/* arcs are created in pairs, so the reverse of arc a is a ^ 1 */
static int64_t dinic(net_t *g, uint32_t s, uint32_t t) {
  int64_t flow = 0;
  int32_t *level = (int32_t *)malloc((size_t)g->N * sizeof(int32_t));
  uint32_t *queue = (uint32_t *)malloc((size_t)g->N * sizeof(uint32_t));
  uint64_t *it = (uint64_t *)malloc((size_t)g->N * sizeof(uint64_t));
  uint64_t *path = (uint64_t *)malloc(((size_t)g->N + 1) * sizeof(uint64_t));
  if (!level || !queue || !it || !path) { flow = -1; goto out; }
  for (;;) {
    for (uint32_t i = 0; i < g->N; i++) level[i] = -1;
    uint32_t qh = 0, qt = 0;
    level[s] = 0;
    queue[qt++] = s;
    while (qh < qt) {
      uint32_t u = queue[qh++];
      for (uint64_t i = g->head[u]; i < g->head[u + 1]; i++) {
        uint64_t a = g->arcs[i];
        if (g->cap[a] > 0 && level[g->to[a]] < 0) {
          level[g->to[a]] = level[u] + 1;
          queue[qt++] = g->to[a];
        }
      }
    }
    if (level[t] < 0) break;
    for (uint32_t i = 0; i < g->N; i++) it[i] = g->head[i];
    uint32_t depth = 0, u = s;
    for (;;) {
      if (u == t) {
        int64_t b = INT64_MAX;
        uint32_t cut = 0;
        for (uint32_t i = 0; i < depth; i++)
          if (g->cap[path[i]] < b) { b = g->cap[path[i]]; cut = i; }
        for (uint32_t i = 0; i < depth; i++) { g->cap[path[i]] -= b; g->cap[path[i] ^ 1] += b; }
        flow += b;
        depth = cut;  /* retreat to the tail of the first saturated arc */
        u = depth ? g->to[path[depth - 1]] : s;
        continue;
      }
      int advanced = 0;
      while (it[u] < g->head[u + 1]) {
        uint64_t a = g->arcs[it[u]];
        uint32_t w = g->to[a];
        if (g->cap[a] > 0 && level[w] == level[u] + 1) {
          path[depth++] = a;
          u = w;
          advanced = 1;
          break;
        }
        it[u]++;
      }
      if (advanced) continue;
      level[u] = -1;  /* dead end */
      if (depth == 0) break;
      depth--;
      u = depth ? g->to[path[depth - 1]] : s;
      it[u]++;
    }
  }
out:
  free(level); free(queue); free(it); free(path);
  return flow;
}

/* nodes that can reach t in the residual graph; the rest is the maximal
 * min-cut source side */
static int reach_sink(const net_t *g, uint32_t t, uint8_t *reach) {
  uint32_t *queue = (uint32_t *)malloc((size_t)g->N * sizeof(uint32_t));
  if (!queue) return -1;
  memset(reach, 0, g->N);
  uint32_t qh = 0, qt = 0;
  reach[t] = 1;
  queue[qt++] = t;
  while (qh < qt) {
    uint32_t w = queue[qh++];
    for (uint64_t i = g->head[w]; i < g->head[w + 1]; i++) {
      uint64_t a = g->arcs[i];      /* w -> u */
      uint32_t u = g->to[a];
      if (!reach[u] && g->cap[a ^ 1] > 0) { reach[u] = 1; queue[qt++] = u; }
    }
  }
  free(queue);
  return 0;
}

static int64_t gcd64(int64_t a, int64_t b) {
  while (b) { int64_t t = a % b; a = b; b = t; }
  return a;
}
/* a/b < c/d for positive denominators */
static int frac_lt(int64_t a, int64_t b, int64_t c, int64_t d) {
  return (__int128)a * d < (__int128)c * b;
}

/* ------------------------------------------------------------------------ */
/* whole pipeline: helpers.cpp:1422-1589                                     */
/* ------------------------------------------------------------------------ */
static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

int oracle_solve(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t k,
                 oracle_result *res, uint8_t *in_set) {
  memset(res, 0, sizeof(*res));
  if (in_set) memset(in_set, 0, n);
  peel_t P;
  if (run_peel(n, off, adj, k, &P)) return -1;
  res->total_cliques = P.m;
  if (P.m == 0 || n == 0) { free_peel(&P); return 0; }

  /* locateDensestCore, helpers.cpp:710-788: the best density over the
   * rows 0..n-1 of the peel table (row 0 = the whole graph), its ceiling
   * k', and the suffix of the removal order from the first row whose
   * removal degree is >= k'. */
  int64_t bn = P.m, bd = n;
  for (uint32_t r = 1; r < n; r++) {
    int64_t a = P.left[r - 1], b = (int64_t)n - r;
    if (frac_lt(bn, bd, a, b)) { bn = a; bd = b; }
  }
  int64_t kp = (bn + bd - 1) / bd;
  res->core_threshold = kp;
  int64_t maxcore = 0;
  for (uint32_t r = 1; r < n; r++)
    if (P.rdeg[r - 1] > maxcore) maxcore = P.rdeg[r - 1];
  res->max_core = maxcore;
  uint32_t index = 1;
  for (; index < n; index++)
    if (P.rdeg[index - 1] >= kp) break;
  uint8_t *incore = (uint8_t *)calloc(n, 1);
  int32_t *cid = (int32_t *)malloc((size_t)n * sizeof(int32_t));  /* component id */
  uint32_t *queue = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
  if (!incore || !cid || !queue) goto fail0;
  for (uint32_t r = index; r <= n; r++) incore[P.order[r - 1]] = 1;
  for (uint32_t v = 0; v < n; v++) res->core_size += incore[v];

  /* core cliques (cliqueEnumerationListRecord, :790-956, re-lists the
   * cliques of the core graph; they are the cliques with every member in
   * the core) */
  int64_t mcore = 0;
  for (int64_t c = 0; c < P.m; c++) {
    int in = 1;
    for (uint32_t j = 0; j < k; j++) in &= incore[P.cl[c * k + j]];
    if (in) {
      if (c != mcore) memmove(P.cl + mcore * k, P.cl + c * k, k * sizeof(uint32_t));
      mcore++;
    }
  }
  res->core_cliques = mcore;

  /* pruneInvalidEdges, :958-993: keep the core edges inside >= 1 clique */
  uint64_t npairs = (uint64_t)mcore * k * (k - 1) / 2;
  uint64_t *pairs = (uint64_t *)malloc((npairs ? npairs : 1) * sizeof(uint64_t));
  if (!pairs) goto fail0;
  uint64_t pi = 0;
  for (int64_t c = 0; c < mcore; c++)
    for (uint32_t i = 0; i < k; i++)
      for (uint32_t j = i + 1; j < k; j++) {
        uint32_t a = P.cl[c * k + i], b = P.cl[c * k + j];
        if (a > b) { uint32_t t = a; a = b; b = t; }
        pairs[pi++] = ((uint64_t)a << 32) | b;
      }
  qsort(pairs, (size_t)pi, sizeof(uint64_t), cmp_u64);
  uint64_t ne = 0;
  for (uint64_t i = 0; i < pi; i++)
    if (i == 0 || pairs[i] != pairs[i - 1]) pairs[ne++] = pairs[i];
  res->pruned_edges = (int64_t)ne;
  /* pruned graph as CSR (both directions) */
  uint64_t *poff = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  uint32_t *padj = (uint32_t *)malloc((2 * ne + 1) * sizeof(uint32_t));
  uint64_t *pcur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  if (!poff || !padj || !pcur) { free(pairs); free(poff); free(padj); free(pcur); goto fail0; }
  for (uint64_t i = 0; i < ne; i++) { poff[(pairs[i] >> 32) + 1]++; poff[(uint32_t)pairs[i] + 1]++; }
  for (uint32_t v = 0; v < n; v++) poff[v + 1] += poff[v];
  memcpy(pcur, poff, ((size_t)n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < ne; i++) {
    uint32_t a = (uint32_t)(pairs[i] >> 32), b = (uint32_t)pairs[i];
    padj[pcur[a]++] = b;
    padj[pcur[b]++] = a;
  }
  free(pcur);
  free(pairs);

  /* connectedComponentDecompose, :995-1116: BFS from every unvisited core
   * vertex in ascending id order; isolated core vertices are components */
  int32_t ncomp = 0;
  for (uint32_t v = 0; v < n; v++) cid[v] = -1;
  for (uint32_t v = 0; v < n; v++) {
    if (!incore[v] || cid[v] >= 0) continue;
    uint32_t qh = 0, qt = 0;
    cid[v] = ncomp;
    queue[qt++] = v;
    while (qh < qt) {
      uint32_t u = queue[qh++];
      for (uint64_t e = poff[u]; e < poff[u + 1]; e++)
        if (cid[padj[e]] < 0) { cid[padj[e]] = ncomp; queue[qt++] = padj[e]; }
    }
    ncomp++;
  }
  free(poff);
  free(padj);
  res->n_components = ncomp;

  /* per-component vertex lists (ascending) and clique lists */
  uint32_t *csize = (uint32_t *)calloc((size_t)ncomp + 1, sizeof(uint32_t));
  int64_t *ccl = (int64_t *)calloc((size_t)ncomp + 1, sizeof(int64_t));
  uint32_t *local = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
  if (!csize || !ccl || !local) { free(csize); free(ccl); free(local); goto fail0; }
  for (uint32_t v = 0; v < n; v++)
    if (cid[v] >= 0) local[v] = csize[cid[v]]++;
  for (int64_t c = 0; c < mcore; c++) ccl[cid[P.cl[c * k]]]++;

  /* dynamicExact, :1120-1254.  The starting answer is the component of
   * largest density (first on ties); later components replace it only with
   * a strictly denser set. */
  int32_t best_c = 0;
  int64_t best_n = ccl[0], best_d = csize[0];
  for (int32_t c = 1; c < ncomp; c++)
    if (frac_lt(best_n, best_d, ccl[c], csize[c])) { best_n = ccl[c]; best_d = csize[c]; best_c = c; }
  uint8_t *best_set = (uint8_t *)calloc(n, 1);
  uint8_t *cur_set = (uint8_t *)calloc(n, 1);
  if (!best_set || !cur_set) { free(best_set); free(cur_set); free(csize); free(ccl); free(local); goto fail0; }
  for (uint32_t v = 0; v < n; v++) best_set[v] = cid[v] == best_c;

  for (int32_t c = 0; c < ncomp; c++) {
    if (ccl[c] == 0) continue;
    uint32_t nc = csize[c];
    int64_t mc = ccl[c];
    uint32_t *verts = (uint32_t *)malloc((size_t)nc * sizeof(uint32_t));
    uint32_t *cm = (uint32_t *)malloc((size_t)mc * k * sizeof(uint32_t));
    int64_t *deg = (int64_t *)calloc(nc, sizeof(int64_t));
    uint8_t *reach = NULL;
    if (!verts || !cm || !deg) { free(verts); free(cm); free(deg); goto fail1; }
    for (uint32_t v = 0; v < n; v++)
      if (cid[v] == c) verts[local[v]] = v;
    int64_t ci = 0;
    for (int64_t q = 0; q < mcore; q++)
      if (cid[P.cl[q * k]] == c) {
        for (uint32_t j = 0; j < k; j++) {
          uint32_t l = local[P.cl[q * k + j]];
          cm[ci * k + j] = l;
          deg[l]++;
        }
        ci++;
      }
    int64_t an = best_n, ad = best_d;
    int improved = 0;
    for (;;) {
      int64_t g = gcd64(an, ad);
      int64_t p = an / g, q = ad / g;
      net_t net;
      memset(&net, 0, sizeof(net));
      if (build_net(&net, nc, mc, k, cm, deg, p, q)) { free_net(&net); goto fail2; }
      uint32_t s = nc + (uint32_t)mc, t = s + 1;
      int64_t f = dinic(&net, s, t);
      res->flows++;
      if (f < 0) { free_net(&net); goto fail2; }
      free(reach);
      reach = (uint8_t *)malloc(net.N);
      if (!reach || reach_sink(&net, t, reach)) { free_net(&net); goto fail2; }
      free_net(&net);
      if (f == q * (int64_t)k * mc) break;  /* saturated: nothing denser than alpha */
      /* the maximal min-cut source side has density > alpha */
      memset(cur_set, 0, n);
      int64_t sz = 0, cnt = 0;
      for (uint32_t l = 0; l < nc; l++)
        if (!reach[l]) { cur_set[verts[l]] = 1; sz++; }
      for (int64_t q2 = 0; q2 < mc; q2++) {
        int in = 1;
        for (uint32_t j = 0; j < k; j++) in &= !reach[cm[q2 * k + j]];
        cnt += in;
      }
      if (sz == 0 || !frac_lt(an, ad, cnt, sz)) goto fail2;  /* cannot happen */
      an = cnt;
      ad = sz;
      improved = 1;
    }
    if (improved) {
      /* saturated at alpha = rho*: the maximal min-cut source side is the
       * maximal densest set of this component */
      memset(best_set, 0, n);
      int64_t sz = 0;
      for (uint32_t l = 0; l < nc; l++)
        if (!reach[l]) { best_set[verts[l]] = 1; sz++; }
      int64_t cnt = 0;
      for (int64_t q2 = 0; q2 < mc; q2++) {
        int in = 1;
        for (uint32_t j = 0; j < k; j++) in &= !reach[cm[q2 * k + j]];
        cnt += in;
      }
      if (cnt * ad != an * sz) goto fail2;  /* cannot happen */
      best_n = cnt;
      best_d = sz;
    }
    free(reach); free(verts); free(cm); free(deg);
    continue;
  fail2:
    free(reach); free(verts); free(cm); free(deg);
    goto fail1;
  }
  res->num = best_n;
  res->den = best_d;
  if (in_set) memcpy(in_set, best_set, n);
  free(best_set); free(cur_set); free(csize); free(ccl); free(local);
  free(incore); free(cid); free(queue);
  free_peel(&P);
  return 0;
fail1:
  free(best_set); free(cur_set); free(csize); free(ccl); free(local);
fail0:
  free(incore); free(cid); free(queue);
  free_peel(&P);
  return -1;
}
