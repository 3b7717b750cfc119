/*
 * everest_b200.h -- C ABI of the B200 temporal-motif miner.
 *
 * Plain pointers, sizes and int status codes; no C++ or torch types cross
 * this boundary.  Every entry point returns EVX_OK (0) or a negative
 * EVX_ERR_* code; evx_last_error() gives a thread-local message for the last
 * failure.  No entry point exits the process (the reference's gpuErrchk
 * calls exit(), include/helpers.cuh:7-15; this layer reports instead).
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the reference project root).
 */
#ifndef EVEREST_B200_H_
#define EVEREST_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define EVX_API __attribute__((visibility("default")))
#else
#define EVX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define EVX_OK 0
#define EVX_ERR_INVALID (-1)   /* bad argument, bad motif, bad sizes */
#define EVX_ERR_CUDA (-2)      /* CUDA runtime error */
#define EVX_ERR_NOMEM (-3)     /* device or host allocation failed / not admitted */
#define EVX_ERR_OVERFLOW (-4)  /* t + delta overflows int32, or sizes exceed int32 ids */
#define EVX_ERR_IO (-5)        /* file missing or unreadable */
#define EVX_ERR_STATE (-6)     /* call out of order (e.g. run before take) */
#define EVX_ERR_TIMEOUT (-7)   /* a bounded device wait gave up */
#define EVX_ERR_NODEVICE (-8)  /* no CUDA device */
#define EVX_ERR_LIMIT (-9)     /* a query passed its work limit (evx_*_set_limit) */

/* Largest motif the kernels are instantiated for. */
#define EVX_MAX_MOTIF_EDGES 8
#define EVX_MAX_MOTIF_NODES 9

/* evx_worker_take flags */
#define EVX_FLAG_STRICT_TS 1u    /* additionally require t(e_j) > t(e_{j-1}) */
#define EVX_FLAG_EXACT_TOTAL 2u  /* enumerate: keep counting past the cap */
#define EVX_FLAG_NO_STEAL 4u     /* disable intra-warp work stealing */
#define EVX_FLAG_NO_PAIR_INDEX 8u /* count the last edge by scanning, not range arithmetic */
/* A closing last edge whose pair changes with every partial match is counted
 * by one pair hash-table lookup per partial match by default; these select
 * the per-node pair directory, or a scan of the shorter endpoint list. */
#define EVX_FLAG_PAIR_DIR 16u
#define EVX_FLAG_CLOSING_SCAN 32u
/* Before scanning the candidates for the second-to-last edge, a search
 * checks that the closing edge's fixed endpoint still has an edge inside the
 * window (and skips the scan when not); this turns that check off. */
#define EVX_FLAG_NO_CLOSING_PRUNE 64u
/* A last edge that maps a new node is scanned four records per lane per
 * step; when its window goes on past that, the rest is counted by range
 * arithmetic (window length minus the entries of the pairs to nodes already
 * mapped).  This keeps the scan instead. */
#define EVX_FLAG_NEW_SCAN 128u
/* A motif edge between two nodes mapped before it (not counted by range
 * arithmetic) walks the run of its static edge (u, v) in the pair index:
 * only the matching edges, after the previous edge and inside the window.
 * This scans the shorter of out(u) / in(v) instead, as the reference does
 * (system/templates/common/resolveMi.snp:9-28). */
#define EVX_FLAG_LIST_SCAN 256u
/* When the last motif edge has a root node as an endpoint, each root's
 * window ends at that node's last entry inside it (a root with none is
 * skipped); this keeps the plain window (same results, for timing). */
#define EVX_FLAG_NO_ROOT_BOUND 2048u
/* evx_worker_take_constrained: a query without anti-edges or a filter (node
 * and edge predicates, temporal gaps) runs on the warp-synchronous search;
 * EVX_FLAG_PER_LANE sends it to the per-lane search instead.
 * EVX_FLAG_WARP_SYNC asks for the warp-synchronous search, the default. */
#define EVX_FLAG_PER_LANE 512u
#define EVX_FLAG_WARP_SYNC 1024u

typedef struct evx_graph evx_graph;   /* a graph resident on one device */
typedef struct evx_worker evx_worker; /* per-device search worker */

/* Thread-local message describing the last failure. */
EVX_API const char *evx_last_error(void);

/* Number of visible CUDA devices (0 when none). */
EVX_API int evx_device_count(int *count);

/* Free and total device memory in bytes (admission of enumeration buffers). */
EVX_API int evx_device_mem_info(int device, int64_t *free_bytes, int64_t *total_bytes);

/* ------------------------------------------------------------ host data --
 * Edge-list loading (replaces EdgeListLoader::createEdgeListCache,
 * src/core/cpu/data.cc:175-290): parse "u v t" lines with atoi semantics,
 * stable-sort by t.  On success *u, *v, *t, *ids hold malloc'd arrays of
 * *num_edges ints (ids = original 0-based line index of each sorted edge);
 * release them with evx_free. */
EVX_API int evx_edgelist_parse(const char *path, int64_t *num_edges,
                       int **u, int **v, int **t, int **ids);

/* Graph building (replaces GraphDataLoader::createGraphData,
 * src/core/gpu/data.cu:124-348): relabels vertices to 0..V-1, builds
 * out/in edge-id lists grouped by endpoint and ascending in edge id, CSR
 * offsets and the AoS {u,v,t} array.  Inputs are the sorted edge range
 * [beg, end) of an edge list.  Outputs are malloc'd (evx_free):
 *   eg[3*E], out_v[E], in_v[E], out_r[V+1], in_r[V+1], euid[E]. */
EVX_API int evx_graph_build_host(const int *u, const int *v, const int *t,
                         const int *ids, int64_t beg, int64_t end,
                         int64_t *num_edges, int64_t *num_vertices,
                         int **eg, int **out_v, int **in_v,
                         int **out_r, int **in_r, int **euid);

/* Motif decoding (replaces HostMotifData::HostMotifData,
 * src/core/cpu/data.cc:411-449 with TemporalGraph::ReadGraph,
 * src/core/cpu/Graph.cc:198-258): lines "u v t", stable-sorted by t, nodes
 * relabeled by first appearance.  Writes k relabeled edges into mu/mv
 * (capacity EVX_MAX_MOTIF_EDGES each) and the node count. */
EVX_API int evx_motif_parse(const char *path, int *k, int *mu, int *mv, int *num_nodes);
EVX_API int evx_motif_parse_text(const char *text, int *k, int *mu, int *mv, int *num_nodes);

EVX_API void evx_free(void *p);

/* Page-lock host memory so uploads from it run as asynchronous DMA
 * (cudaHostRegister / cudaHostUnregister). */
EVX_API int evx_host_register(void *ptr, int64_t bytes);
EVX_API int evx_host_unregister(void *ptr);

/* --------------------------------------------------------- device graph --
 * Allocation + host->device transfer of one graph (replaces
 * GraphDataManager::alloc / moveAsync / waitMove,
 * src/core/gpu/data.cu:380-467, and DeviceGraphData, include/data.h:239-247).
 * Inputs are host arrays in the layout evx_graph_build_host produces; they
 * may be pageable or pinned.  The device-side packed layout (16-byte
 * adjacency records) is built on the device from them.  stream may be NULL
 * (the worker-independent upload stream is used). */
EVX_API int evx_graph_upload(int device, int64_t num_edges, int64_t num_vertices,
                     const int *eg, const int *out_v, const int *in_v,
                     const int *out_r, const int *in_r, const int *euid,
                     void *stream, evx_graph **out);

/* Same, from device-resident inputs (no host copy). */
EVX_API int evx_graph_from_device(int device, int64_t num_edges, int64_t num_vertices,
                          const int *eg_d, const int *out_v_d, const int *in_v_d,
                          const int *out_r_d, const int *in_r_d, const int *euid_d,
                          void *stream, evx_graph **out);

EVX_API int evx_graph_free(evx_graph *g);
EVX_API int evx_graph_info(const evx_graph *g, int64_t *num_edges, int64_t *num_vertices,
                   int *device, int64_t *device_bytes);

/* --------------------------------------------------------------- worker --
 * Worker construction (replaces the plugin factory getWorker(int gpu),
 * system/templates/GPUWorker/interface.snp:1-7, and the worker ctor,
 * system/templates/GPUWorker/ctor.snp).  stream: cudaStream_t to launch on,
 * or NULL to create one owned by the worker. */
EVX_API int evx_worker_create(int device, void *stream, evx_worker **out);
EVX_API int evx_worker_destroy(evx_worker *w);
EVX_API int evx_worker_stream(evx_worker *w, void **stream);

/* Bind a job (replaces DeviceJobData ctor, src/core/gpu/data.cu:496-529,
 * MineJob, src/core/cpu/data.cc:452-466, and GPUWorker::take,
 * system/templates/GPUWorker/take.snp).  mu/mv: k relabeled motif edges
 * (edge 0 = (0,1); each later edge touches a mapped node; no self-loops).
 * Roots are edge ids [beg, end); end < 0 means E-k+1.  enum_cap > 0 selects
 * enumeration with that many rows of k ints (the YAML enumerate: <cap>).
 * Fails with EVX_ERR_OVERFLOW if max(t) + delta overflows int32 and with
 * EVX_ERR_NOMEM if the enumeration buffer does not fit in free memory. */
EVX_API int evx_worker_take(evx_worker *w, const evx_graph *g, int k, const int *mu,
                    const int *mv, int delta, int64_t beg, int64_t end,
                    int64_t enum_cap, unsigned flags);

/* Run the bound job to completion and return the count (replaces
 * GPUWorker::run, system/templates/GPUWorker/run.snp, and the generated
 * TMotifMatchingGPUImpl, system/templates/Impl/top.snp).  In count mode the
 * result is the exact match count; in enumerate mode it is the number of
 * matches found before root dispatch stopped at the cap (exact total with
 * EVX_FLAG_EXACT_TOTAL). */
EVX_API int evx_worker_run(evx_worker *w, uint64_t *count);

/* Asynchronous form of evx_worker_run: enqueue the search on the worker's
 * stream; evx_worker_result synchronises and returns the count. */
EVX_API int evx_worker_launch(evx_worker *w);
EVX_API int evx_worker_result(evx_worker *w, uint64_t *count);
/* *done = 1 when the launched search has finished (never blocks). */
EVX_API int evx_worker_query(evx_worker *w, int *done);

/* Copy min(n, rows found, cap) enumeration rows (k ints each: the original
 * line ids of e_0..e_{k-1}) to host memory (replaces
 * GPUWorker::printEnum, system/templates/enumerate/func.snp). */
EVX_API int evx_worker_enum_rows(evx_worker *w, int64_t n, int *rows, int64_t *rows_written);

/* Tuning knobs (autotuner): block size, blocks per SM (0 = occupancy),
 * roots per warp fetch, steal check interval (iterations, 0 = never),
 * minimum range width worth splitting. */
EVX_API int evx_worker_set_tuning(evx_worker *w, int block, int blocks_per_sm,
                          int roots_per_fetch, int steal_interval, int min_split);

/* Kernel statistics of the last run: launches of this library's kernels
 * and device milliseconds measured with CUDA events around them. */
EVX_API int evx_worker_last_stats(evx_worker *w, int *kernel_launches, float *device_ms);

/* Work limit for later jobs of this worker (0 = none, the default).  No
 * counterpart in the reference, whose searches always run to the end.  A
 * serving caller uses it to bound the work of any one query.  The work
 * measure ("meter") is the number of adjacency records the search examines
 * inside their time windows; every such record is examined exactly once
 * however the scans are split between lanes, so the meter is fixed by the
 * graph and the query, not by scheduling.  Once the meter is known to
 * exceed max_work the search stops, and evx_worker_run / evx_worker_result
 * return EVX_ERR_LIMIT with *count set to the matches counted so far (a
 * lower bound; an enumeration keeps the rows written so far, readable with
 * evx_worker_enum_rows).  A query whose meter stays <= max_work is never
 * stopped and its result is exact, so whether a query is stopped does not
 * depend on scheduling. */
EVX_API int evx_worker_set_limit(evx_worker *w, uint64_t max_work);

/* -------------------------------------------------------------- batches --
 * Many count queries against one resident graph in one persistent launch
 * per motif size (no counterpart in the reference, whose batch driver
 * re-generates, re-compiles and re-launches per query,
 * system/batch-query.py:14-20 and system/tmine/frontend.py:135-143).  The
 * root ranges of a size's queries are cut into tiles that form one device
 * work queue.  The launch sequence is captured in a CUDA graph and replayed
 * while the batch keeps its shape. */
typedef struct evx_batch evx_batch;
EVX_API int evx_batch_create(int device, int max_queries, void *stream, evx_batch **out);
EVX_API int evx_batch_destroy(evx_batch *b);
/* Add one count query (all queries of a batch use one graph); *index = its
 * position in the result array. */
EVX_API int evx_batch_add(evx_batch *b, const evx_graph *g, int k, const int *mu, const int *mv,
                          int delta, int64_t beg, int64_t end, unsigned flags, int *index);
EVX_API int evx_batch_clear(evx_batch *b);
EVX_API int evx_batch_launch(evx_batch *b);
/* Wait for the launched batch; counts[i] for the first n queries. */
EVX_API int evx_batch_result(evx_batch *b, uint64_t *counts, int n);
EVX_API int evx_batch_run(evx_batch *b, uint64_t *counts, int n);
/* *done = 1 when the launched batch has finished (never blocks). */
EVX_API int evx_batch_query(evx_batch *b, int *done);
/* tile_roots (multiple of 32), blocks per SM (0 = occupancy), steal
 * interval, min split, use_graph (capture + replay), reserved. */
EVX_API int evx_batch_set_tuning(evx_batch *b, int tile_roots, int blocks_per_sm, int steal_interval,
                                 int min_split, int use_graph, int reserved);
EVX_API int evx_batch_last_stats(evx_batch *b, int *kernel_launches, float *device_ms);

/* Work limit per query of this batch (0 = none): evx_worker_set_limit's
 * rule, query by query.  evx_batch_result still returns EVX_OK; it writes
 * UINT64_MAX as the count of each stopped query and the exact count of
 * every other query. */
EVX_API int evx_batch_set_limit(evx_batch *b, uint64_t max_work);

/* ------------------------------------------------- allocation-free count --
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * at query time (device memory fully reserved by another allocator, or a
 * device with no free memory left): runs nq count queries (1 <=
 * nq <= EVX_STATIC_MAX_QUERIES) on a resident graph and writes the counts to
 * counts[nq] (host memory), with no cudaMalloc / cudaFree / allocating call.
 * Its scratch is a file-scope device array of EVX_STATIC_MAX_QUERIES slots
 * (4 KB per device, held until the process exits).  Query q is motif edges
 * mu/mv[off_q .. off_q + k[q]) with off_q = k[0] + ... + k[q-1], window
 * delta[q]; roots are [beg, end) (end < 0: E - k + 1).  The first call on a
 * device looks up the array's device address, so it must come before any
 * stream capture.  All calls share the array: calls whose GPU work overlaps
 * race, so serialise them.  Rejects nq > EVX_STATIC_MAX_QUERIES.  Every
 * query is checked before the first launch (an error for a bad query leaves
 * nothing queued); the call returns once the counts are in host memory (it
 * waits for `stream`), and it leaves the caller's current device as it was. */
#define EVX_STATIC_MAX_QUERIES 256
EVX_API int evx_count_static(const evx_graph *g, int nq, const int *k, const int *mu,
                             const int *mv, const int *delta, int64_t beg, int64_t end,
                             unsigned flags, void *stream, uint64_t *counts);

/* ---------------------------------------------------------- constraints --
 * Replaces the reference's per-query generated constraint code
 * (system/tmine/Query.py:39-310 renders C snippets that KernelGen.py:288-336,
 * 467-533 and system/templates/common/{nextMatchInTask,structuralConstraint,
 * lookAtMatchRes,findMatch}.snp compile into each plugin).  Here one
 * precompiled kernel reads the constraints as data:
 *
 *   node predicates  (YAML `node: <expr in f>` or `node0..node{n-1}`): f is
 *                    the node feature of the graph node a motif node maps to;
 *   edge predicate   (YAML `edge: <expr in f>`): f is the edge feature of
 *                    every matched edge (and of every anti-edge candidate);
 *   temporal         (YAML `temporal: [g_0 .. g_{k-2}]`): motif edge j >= 1
 *                    must have t <= t(previous real edge) + g_{j-1}, and for
 *                    j >= 2 also t <= t(e_0) + delta (delta alone does not
 *                    bound a two-edge motif with a temporal list, as in the
 *                    reference: KernelGen.py:470-476);
 *   anti-edges       (YAML `antiEdge: [bool x k]`): motif edge j must NOT
 *                    exist: a partial match is dropped when some edge after
 *                    the previous real edge, inside that edge's window, joins
 *                    the two (already mapped) nodes and passes the edge
 *                    predicate (lookAtMatchRes.snp:1-21);
 *   filter           (YAML `filter: <expr in e0, e1, ...>`): e_i is the edge
 *                    feature of the edge matched to motif edge i, evaluated
 *                    once per complete match (findMatch.snp:1-8).
 *
 * Expressions are C integer expressions compiled to a postfix program: each
 * instruction is op[i] | EVX_OP_WRAP32 (the result is an int: wrap it to 32
 * bits) with arg[i] the constant or the variable index.  Values are int64;
 * comparisons and logical operators give 0 or 1; division or remainder by
 * zero gives 0; shifts use the count modulo the operand width. */
#define EVX_PROG_MAX 48
#define EVX_OP_CONST 1   /* push arg */
#define EVX_OP_VAR 2     /* push variable arg (f = 0; e_i = i) */
#define EVX_OP_NEG 3
#define EVX_OP_NOT 4     /* logical ! */
#define EVX_OP_BNOT 5    /* ~ */
#define EVX_OP_ADD 6
#define EVX_OP_SUB 7
#define EVX_OP_MUL 8
#define EVX_OP_DIV 9
#define EVX_OP_MOD 10
#define EVX_OP_SHL 11
#define EVX_OP_SHR 12
#define EVX_OP_LT 13
#define EVX_OP_LE 14
#define EVX_OP_GT 15
#define EVX_OP_GE 16
#define EVX_OP_EQ 17
#define EVX_OP_NE 18
#define EVX_OP_BAND 19
#define EVX_OP_BXOR 20
#define EVX_OP_BOR 21
#define EVX_OP_LAND 22
#define EVX_OP_LOR 23
#define EVX_OP_COND 24   /* c ? a : b, pushed c, a, b */
#define EVX_OP_WRAP32 0x80
#define EVX_PROG_STACK 16

typedef struct evx_program {
  int32_t len;                 /* instructions (0 = always true) */
  int32_t op[EVX_PROG_MAX];
  int64_t arg[EVX_PROG_MAX];
} evx_program;

typedef struct evx_constraints {
  uint32_t anti_mask;          /* bit j: motif edge j is an anti-edge */
  int32_t has_temporal;
  int32_t temporal[EVX_MAX_MOTIF_EDGES - 1];
  int32_t node_mode;           /* 0 none, 1 node[0] for every node, 2 node[a] for motif node a */
  evx_program node[EVX_MAX_MOTIF_NODES];
  int32_t has_edge;
  evx_program edge;
  int32_t has_filter;
  evx_program filter;
} evx_constraints;

/* Node features (int32 per graph vertex id) and edge features (int32 per
 * sorted edge id) of a resident graph; either may be NULL (kept as before).
 * Host arrays, copied to the graph's device on the legacy default stream.
 * Set them before taking constrained jobs on the graph, not while one is
 * taken or running: a job's predicate masks are built from the features
 * when it is taken, and its filter reads the edge features while it runs,
 * so a change in between would mix old and new values. */
EVX_API int evx_graph_set_features(evx_graph *g, const int *node_features, const int *edge_features);

/* evx_worker_take with constraints (c may be NULL: plain search).  Checks
 * what the reference cannot run: an anti-edge as motif edge 0, 1 or k-1
 * (the generated search never ends or reads past its arrays there), an
 * anti-edge touching a node that no earlier real edge maps, a filter naming
 * an anti-edge, and enumeration with anti-edges (its rows would name no
 * edge); node / edge predicates need the matching features on the graph.
 * Flags: EVX_FLAG_EXACT_TOTAL, EVX_FLAG_PER_LANE and EVX_FLAG_WARP_SYNC
 * only.  A query without anti-edges or a filter runs on the
 * warp-synchronous search with the checks compiled in (the per-lane
 * constrained search with EVX_FLAG_PER_LANE); anti-edges or a filter take
 * the per-lane constrained search.  The plain search's launch, result and rows
 * calls then run this job; the work limit (evx_worker_set_limit) does not
 * apply to it.  A struct with no constraint set runs the plain search. */
EVX_API int evx_worker_take_constrained(evx_worker *w, const evx_graph *g, int k, const int *mu,
                                        const int *mv, int delta, int64_t beg, int64_t end,
                                        int64_t enum_cap, unsigned flags, const evx_constraints *c);

#ifdef __cplusplus
}
#endif
#endif /* EVEREST_B200_H_ */
