/* cds.h -- C ABI of the B200 k-clique densest-subgraph engine (libcds).
 *
 * The reference (wajidmanzoor/CDS) has no library API: its surface is the
 * command line `./main <graph> <k> <pSize> <cpSize> <glBufferSize>
 * <partitionSize> <earlyStop>` (cudaCode/main.cu:865-887) over stage
 * functions that share global device structs (cudaCode/main.cu:22-863,
 * cudaCode/inc/common.h:47-143).  Each entry point below names the stage of
 * the reference it replaces.  The CLI built on top of this header
 * (cds_b200/bin/main) keeps the reference's arguments and output keys.
 *
 * Conventions
 *  - Every function returns cds_status; nothing calls exit() and no C++
 *    exception crosses this boundary.  cds_last_error() returns the text of
 *    the last failure on a context.
 *  - A cds_ctx owns one CUDA device, its streams and a stream-ordered device
 *    memory pool capped at cds_config.mem_budget bytes.  A context is used
 *    by one host thread at a time, except through the server calls, which
 *    are thread-safe.
 *  - All counts are exact 64-bit integers.  A density is reported as the
 *    exact fraction num/den = (k-cliques inside the set) / (set size).
 *  - Host arrays passed in are copied; arrays handed out are owned by the
 *    library and released with the matching *_free call.
 */
#ifndef CDS_H
#define CDS_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cds_status {
  CDS_OK = 0,
  CDS_ERR_OOM = 1,       /* device memory budget or allocation exhausted     */
  CDS_ERR_OVERFLOW = 2,  /* a count exceeds the engine's index width         */
  CDS_ERR_TIMEOUT = 3,   /* a device loop hit its iteration budget           */
  CDS_ERR_INPUT = 4,     /* malformed graph, file or argument                */
  CDS_ERR_CUDA = 5,      /* CUDA runtime error                               */
  CDS_ERR_STATE = 6,     /* call not valid in the current state              */
  CDS_ERR_NOT_READY = 7  /* cds_poll: the request is still running          */
} cds_status;

typedef struct cds_ctx cds_ctx;
typedef struct cds_graph cds_graph;
typedef struct cds_server cds_server;

typedef struct cds_config {
  int device;           /* CUDA device ordinal                                */
  uint64_t mem_budget;  /* bytes of device memory the context may hold;
                           0 = 90% of the device's free memory at creation    */
  uint32_t streams;     /* worker streams for batches and serving (0 = 4;
                           at most CDS_MAX_INFLIGHT, else CDS_ERR_INPUT)      */
  uint32_t flags;       /* CDS_CONFIG_* bits, 0 for the defaults              */
} cds_config;

/* cds_config.flags.  No counterpart in the reference (its layouts are fixed). */
/* The peel reads clique ids and gathers member records instead of streaming
 * per-incidence copies of the other members: (k-1)x less peel memory for
 * k <= 4 (the default falls back to it only when the copies do not fit),
 * slower sweeps. */
#define CDS_CONFIG_COMPACT_PEEL 1u
/* 64-bit clique indices in the incidence lists and 64-bit flow state in
 * every flow network, whatever its size (the default narrows them to 32
 * bits when they fit). */
#define CDS_CONFIG_WIDE_FLOW 2u
/* 64-bit clique ids in the peel's clique-id layout, whatever the count (a
 * listing of 2^32 or more cliques always uses them; member layouts need no
 * clique ids).  Implies the clique-id layout. */
#define CDS_CONFIG_WIDE_CLIQUE_IDS 4u

/* Solve parameters: the reference CLI's positional arguments
 * (cudaCode/main.cu:870-887) plus the search policy. */
typedef struct cds_params {
  uint32_t k;               /* clique size, 2..CDS_MAX_K                       */
  uint32_t p_size;          /* pSize: listing work-buffer entries per warp     */
  uint32_t cp_size;         /* cpSize: staged cliques per warp before a flush  */
  uint32_t gl_buffer_size;  /* glBufferSize: peel removal-buffer entries/block */
  uint32_t partition_size;  /* partitionSize: active-node queue entries per
                               flow network                                    */
  int32_t early_stop;       /* -1: exact.  >= 0: stop a max-flow after this
                               many global-relabel cycles without sink
                               progress (approximate, opt-in)                  */
  uint32_t search;          /* CDS_SEARCH_*: how the answer is found         */
} cds_params;

/* cds_params.search.  The exact searches return the optimum (ub = answer);
 * CDS_SEARCH_CORE returns the densest (k,Psi)-core that the peel finds --
 * the CoreApp answer, the "Densest Core Density" the reference prints
 * (cudaCode/main.cu:1071) -- with no flow at all: a real vertex set with its
 * exact density, approximate, its gap shown by ub_num/ub_den. */
#define CDS_SEARCH_DINKELBACH 0u  /* binary search on alpha, Dinkelbach re-centring */
#define CDS_SEARCH_BISECT 1u      /* plain bisection on the grid j / (n_c (n_c-1))  */
#define CDS_SEARCH_CORE 2u        /* approximate: the densest core                   */

#define CDS_MAX_K 16
#define CDS_MAX_INFLIGHT 64  /* worker streams of a context and server workers, at most */

enum {
  CDS_T_DAG = 0,
  CDS_T_LIST,
  CDS_T_PEEL,
  CDS_T_CORE,
  CDS_T_PRUNE,
  CDS_T_COMPONENTS,
  CDS_T_EXACT,
  CDS_T_TOTAL,
  CDS_T_COUNT
};

typedef struct cds_result {
  uint64_t num, den;         /* density of the answer = num/den               */
  uint64_t total_cliques;    /* |Psi| of the whole graph                      */
  uint64_t max_core;         /* largest (k,Psi)-clique-core number            */
  uint64_t core_threshold;   /* k' = ceil(best core density)                  */
  uint64_t core_num, core_den;  /* best core density (exact fraction)         */
  uint64_t core_size;        /* vertices of the (k',Psi)-core                 */
  uint64_t core_cliques;     /* k-cliques inside that core                    */
  uint64_t pruned_edges;     /* core edges that lie in >= 1 core clique       */
  uint32_t n_components;     /* connected components of the pruned core       */
  uint32_t flows;            /* max-flow solves performed                     */
  uint32_t early_stopped;    /* 1 if early_stop cut a max-flow short          */
  uint32_t peel_levels;      /* distinct levels the peel went through         */
  double t_ms[CDS_T_COUNT];  /* stage times (device events), milliseconds     */
  uint64_t size;             /* answer size (= den, or 0 when |Psi| = 0)      */
  uint32_t *vertices;        /* answer vertices, ascending (library-owned)    */
  /* proven upper bound of the optimum density: equal to num/den for an exact
   * answer; for an approximate one (early_stop cut a flow short, or
   * CDS_SEARCH_CORE) the gap to it bounds how far the answer can be off */
  uint64_t ub_num, ub_den;
  /* per component of the pruned core that holds cliques, in order: the
   * search's starting lower bound (the densest whole component) and the
   * bound |Psi_c|^((k-1)/k) / (k!)^(1/k) -- the reference's lb= and ub= lines
   * (cudaCode/main.cu:1092-1103); library-owned, n_bounds entries each */
  uint32_t n_bounds;
  double *bound_lb, *bound_ub;
  double t_queue_ms;         /* server: submission to the start of its batch  */
  double t_service_ms;       /* server: start of its batch to its answer      */
} cds_result;

const char *cds_version(void);
const char *cds_status_string(cds_status s);

/* Context: replaces the global device structs and per-stage cudaMalloc of
 * cudaCode/src/gpuMemoryAllocation.cu:5-225 and cudaCode/src/common.cpp:4-12. */
cds_status cds_create(const cds_config *cfg, cds_ctx **out);
void cds_destroy(cds_ctx *ctx);
const char *cds_last_error(const cds_ctx *ctx);
/* Bytes the context currently holds on the device, and its high-water mark. */
cds_status cds_mem_usage(const cds_ctx *ctx, uint64_t *in_use, uint64_t *peak);

/* Graphs: replace Graph::Graph (cudaCode/src/graph.cpp:7-40) and the CSR
 * upload of memoryAllocationGraph (cudaCode/src/gpuMemoryAllocation.cu:5-50).
 * cds_graph_load_file reads the file's bytes once and parses adjacency-list
 * text on the device (vertex lines in any order, duplicates merged, lists
 * symmetrised, self-loops dropped); a binary CSR cache file
 * (cds_write_csr_binary, cds_gen.h) is uploaded as it is and must hold a
 * canonical CSR.  cds_graph_from_csr expects a symmetric CSR (off[n+1],
 * adj[off[n]]) with ascending rows and no self-loops and checks it. */
cds_status cds_graph_load_file(cds_ctx *ctx, const char *path, cds_graph **out);
cds_status cds_graph_from_csr(cds_ctx *ctx, const uint64_t *off, const uint32_t *adj,
                              uint32_t n, cds_graph **out);
cds_status cds_graph_info(const cds_graph *g, uint32_t *n, uint64_t *m,
                          uint32_t *max_degree);
/* Copies a graph's canonical CSR back to the host: off[n+1], adj[2m] (e.g. to
 * keep a parsed text file as a binary cache, cds_write_csr_binary). */
cds_status cds_graph_download(const cds_graph *g, uint64_t *off, uint32_t *adj);
void cds_graph_free(cds_graph *g);

/* Stage entry points (parity tests and tools). */

/* generateDAG + listAllCliques/countCliques (cudaCode/main.cu:22-250,
 * :919-977 for k = 2): the number of k-cliques and, if clique_degree is not
 * NULL, each vertex's clique degree (n entries), both exact 64-bit counts
 * with no 2^32 cap (the reference keeps them in 32 bits, the CPU program in
 * long: cpuCode/c++/src/helpers.cpp:436-447). */
cds_status cds_list_cliques(cds_ctx *ctx, cds_graph *g, uint32_t k, uint32_t p_size,
                            uint32_t cp_size, uint64_t *count, uint64_t *clique_degree);

/* cliqueCoreDecompose (cudaCode/main.cu:252-343): clique-core number of
 * every vertex (core, n entries), the largest one and |Psi|. */
cds_status cds_clique_core(cds_ctx *ctx, cds_graph *g, uint32_t k,
                           uint32_t gl_buffer_size, uint64_t *core, uint64_t *max_core,
                           uint64_t *count);

/* generateDensestCore (cudaCode/main.cu:345-399): the best core density
 * (num/den), k' = ceil(num/den) and, if in_core is not NULL, membership of
 * the (k',Psi)-core (n bytes). */
cds_status cds_densest_core(cds_ctx *ctx, cds_graph *g, uint32_t k, uint64_t *threshold,
                            uint64_t *num, uint64_t *den, uint8_t *in_core);

/* prune + componentDecompose (cudaCode/main.cu:400-518;
 * cpuCode/c++/src/helpers.cpp:958-1116) after the densest core of
 * cds_densest_core: the k-cliques inside the (k',Psi)-core, the core edges
 * that lie in at least one of them, and the connected components those edges
 * form that hold at least one core clique, in ascending order of their
 * smallest vertex -- first[i] (smallest vertex), size[i] (vertices),
 * cliques[i] (core cliques).  *count receives the number of components; the
 * arrays (cap entries each, any may be NULL) the first min(count, cap). */
cds_status cds_components(cds_ctx *ctx, cds_graph *g, uint32_t k, uint64_t *core_cliques,
                          uint64_t *pruned_edges, uint32_t *count, uint32_t *first,
                          uint64_t *size, uint64_t *cliques, size_t cap);

/* The whole solve (cudaCode/main.cu:895-1107): DAG, listing, peel, densest
 * core, prune, components, max-flow search. */
cds_status cds_solve(cds_ctx *ctx, cds_graph *g, const cds_params *params,
                     cds_result *result);
void cds_result_free(cds_result *result);

/* Batched solve: many independent instances packed into shared launches.
 * results[i] answers jobs[i]; each must be released with cds_result_free. */
typedef struct cds_job {
  cds_graph *graph;
  cds_params params;
} cds_job;
cds_status cds_solve_batch(cds_ctx *ctx, const cds_job *jobs, size_t n,
                           cds_result *results);

/* Serving: worker threads (one per context stream) take submitted requests
 * into batches of the same k and size class and run them on their streams;
 * graphs of at least 2^20 arcs run alone, and with two or more workers one
 * always stays free for smaller requests.  Admission is by device memory:
 * a bound on the graph and listing state before a batch starts, then, once
 * the listing has counted |Psi|, what the clique store, peel and flow
 * networks can take (the worker waits while that does not fit and another
 * batch runs).  A batch that runs out of memory is split and its requests
 * run again alone. */
typedef struct cds_server_config {
  uint32_t max_batch;       /* instances per batch (0 = 64)                   */
  uint64_t mem_budget;      /* device bytes for resident state (0 = context's) */
  uint32_t max_inflight;    /* concurrent batches on the device (0 = streams;
                               at most CDS_MAX_INFLIGHT, else CDS_ERR_INPUT) */
  uint32_t flags;           /* reserved, 0                                     */
} cds_server_config;
cds_status cds_server_start(cds_ctx *ctx, const cds_server_config *cfg, cds_server **out);
/* The graph must stay alive until the request completes. */
cds_status cds_submit(cds_server *s, cds_graph *g, const cds_params *params,
                      uint64_t *ticket);
/* A request on a graph given as a host CSR (as cds_graph_from_csr takes it):
 * the worker that runs it uploads and checks the graph on its own stream and
 * frees it with the answer, so ingestion overlaps other requests' device
 * work.  off and adj must stay alive and unchanged until the request is
 * answered (pinned host memory makes the upload fastest).  A malformed CSR
 * answers CDS_ERR_INPUT for that ticket. */
cds_status cds_submit_csr(cds_server *s, const uint64_t *off, const uint32_t *adj, uint32_t n,
                          const cds_params *params, uint64_t *ticket);
/* CDS_ERR_NOT_READY while the request runs; otherwise its status, with the
 * answer in *result (release with cds_result_free).  A ticket is answered
 * once. */
cds_status cds_poll(cds_server *s, uint64_t ticket, cds_result *result);
cds_status cds_wait(cds_server *s, uint64_t ticket, cds_result *result);
/* Finishes every admitted request, then stops the scheduler. */
cds_status cds_server_stop(cds_server *s);

/* Autotune: times the listing, peel and max-flow launch shapes on sample
 * graphs and keeps the fastest per clique size; results are cached in
 * cache_path (may be NULL) as "k key value" lines and used by later solves
 * on this context.  When the file already holds lines for k they are loaded
 * and nothing is timed (so n = 0 only loads).  Keys: list_warp_block,
 * list_warp_dmax, list_team_block, flow_rounds, flow_block, peel_chunk,
 * flow_warm, peel_order, flow_inc_per_block, peel_static; unknown keys and
 * out-of-range values are ignored.  flow_warm is the number of balancing
 * passes before each max-flow (weight updates, then the split of every
 * clique's units it starts from): 0 none, -1 (the default) three for
 * networks of 2^20 cliques or more and none below. */
cds_status cds_autotune(cds_ctx *ctx, cds_graph *const *graphs, size_t n, uint32_t k,
                        const char *cache_path);

/* k-clique count and clique degrees of a graph already in device memory,
 * written to caller-owned device buffers, with no device memory allocated.
 * No counterpart in the reference (its listing allocates per stage,
 * cudaCode/src/gpuMemoryAllocation.cu:53-93).  For callers that cannot call
 * cudaMalloc mid-work: code under a framework or memory manager that owns
 * all of the device's memory (a caching allocator that reserved it up
 * front, a host with a fixed device budget), where a new allocation would
 * fail or take memory promised elsewhere.  Scratch lives in one static
 * device array of about 21 MiB that every GPU loading libcds keeps until the
 * process exits.
 *   d_off[n+1] (u64), d_adj[d_off[n]] (u32): a symmetric CSR in device memory
 *     with ascending rows and no self-loops; n <= 262,144 vertices,
 *     d_off[n] <= 4,194,304 arcs, out-degree of the degree-ordered DAG
 *     <= 1,024.  Anything else returns CDS_ERR_INPUT.  The check runs on the
 *     device in two steps, each read back before the next kernel runs: the
 *     offsets first (d_off[0] = 0, never decreasing), then the ids (below n,
 *     ascending, each arc with its reverse); no kernel indexes with an id or
 *     offset the check has not passed.
 *   d_count: one u64 (device); d_clique_degree: n u32 (device) or NULL.
 *   stream: a cudaStream_t (NULL = legacy default stream).
 * The first call on a device looks up the array's device address.  Each call
 * waits on the stream several times to read scalars back (the checks, the
 * DAG's size, the listing's status) and returns once the count is complete.
 * All calls share the one array, which keeps the last call's contents: calls
 * whose work overlaps on a GPU (other threads, other streams) race and must
 * be serialised by the caller. */
cds_status cds_count_cliques_noalloc(const uint64_t *d_off, const uint32_t *d_adj, uint32_t n,
                                     uint32_t k, unsigned long long *d_count,
                                     uint32_t *d_clique_degree, void *stream);

/* Kernel profiling: while on, the context brackets each of its main kernel
 * launches with device events on the launching stream.  cds_profile_read
 * writes {"kernel": [launches, total_ms], ...} (JSON) into buf and resets
 * the counters; CDS_ERR_INPUT if len is too small.  Tracing aid with no
 * counterpart in the reference, which times whole stages on the host
 * (cudaCode/main.cu:904-1088). */
cds_status cds_profile(cds_ctx *ctx, int on);
cds_status cds_profile_read(cds_ctx *ctx, char *buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif
