/* cds_gen.h -- seeded synthetic graph generators and adjacency-list I/O.
 *
 * Host-side helpers of libcds (no GPU needed).  Every generator returns a
 * canonical symmetric CSR: rows ascending, no self-loops, no duplicates.
 * Arrays are allocated by the library and released with cds_free().
 *
 * The adjacency-list text format is the reference's (README.md:72-89 of
 * wajidmanzoor/CDS; readers cudaCode/src/graph.cpp:7-40 and
 * cpuCode/c++/src/graph.cpp:9-52): a header line "n m", then one line
 * "v nbr nbr ..." per vertex.
 */
#ifndef CDS_GEN_H
#define CDS_GEN_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Erdos-Renyi G(n, p). */
int cds_gen_er(uint32_t n, double p, uint64_t seed, uint64_t **off, uint32_t **adj);

/* R-MAT with 2^scale slots, edge_factor * 2^scale sampled edges, quadrant
 * probabilities a, b, c (d = 1-a-b-c); vertex ids are randomly permuted.
 * n may be below 2^scale (samples that land on ids >= n are redrawn); pass
 * n = 0 for n = 2^scale. */
int cds_gen_rmat(uint32_t scale, uint32_t n, double edge_factor, double a, double b,
                 double c, uint64_t seed, uint32_t *n_out, uint64_t **off, uint32_t **adj);

/* Adds a community of `size` vertices chosen at random among n, each pair
 * joined with probability p, to a canonical CSR; returns a new CSR.  The
 * chosen vertex ids are written to members[size] when members != NULL. */
int cds_gen_plant(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t size,
                  double p, uint64_t seed, uint64_t **off_out, uint32_t **adj_out,
                  uint32_t *members);

/* Canonicalises an arbitrary edge list (u[i], v[i]) over n vertices:
 * symmetrises, drops self-loops and duplicates, sorts rows. */
int cds_csr_from_edges(uint32_t n, const uint32_t *u, const uint32_t *v, uint64_t m,
                       uint64_t **off, uint32_t **adj);

/* Binary CSR cache file: this header, then off[n+1] (u64) and adj[nnz]
 * (u32), little-endian.  No counterpart in the reference, which re-parses
 * the text on every run (cudaCode/src/graph.cpp:7-40); cds_graph_load_file
 * and cds_read_adjlist recognise it by its magic. */
#define CDS_CSR_MAGIC "CDSCSR\x01\n"
typedef struct cds_csr_header {
  char magic[8];      /* CDS_CSR_MAGIC */
  uint32_t version;   /* 1 */
  uint32_t reserved;  /* 0 */
  uint64_t n;         /* vertices */
  uint64_t nnz;       /* directed arcs = off[n] */
} cds_csr_header;

/* Writes a CSR as a binary cache file. */
int cds_write_csr_binary(const char *path, uint32_t n, const uint64_t *off, const uint32_t *adj);

/* Reads the adjacency-list format, or a binary cache file, into a canonical
 * CSR (rows may come in any order or be missing; lists are symmetrised and
 * de-duplicated). */
int cds_read_adjlist(const char *path, uint32_t *n, uint64_t **off, uint32_t **adj);

/* Writes a canonical CSR in the adjacency-list format (every vertex line
 * present, ascending). */
int cds_write_adjlist(const char *path, uint32_t n, const uint64_t *off, const uint32_t *adj);

void cds_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
