/*
 * d-core-b200 -- C ABI of the B200 (sm_100a) D-core engine.
 *
 * Drop-in boundary for the load -> decompose -> maintain path of
 * llysdal/d-core-cuda.  The reference exposes that path as C++ free functions
 * and classes compiled into one binary with main(); each entry point below
 * names the reference interface it replaces (file:line in the reference tree).
 *
 * Conventions
 *   - Every function returns DC_OK (0) or a negative DC_ERR_* code;
 *     dc_last_error() gives the message of the calling thread's last failure.
 *   - Plain pointers and sizes only.  Host buffers belong to the caller; the
 *     engine owns all device memory of a graph handle.
 *   - Values are the reference's types: `degree` = int32_t
 *     (src/common.h:59), vertex ids and offsets = uint32_t (src/common.h:60-62).
 *   - A graph handle is used by one host thread at a time; distinct handles
 *     may be used from different threads concurrently (each has its own
 *     CUDA stream).
 */
#ifndef DCORE_B200_H
#define DCORE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DC_OK 0
#define DC_ERR_INVALID (-1)   /* bad argument, malformed input            */
#define DC_ERR_CUDA (-2)      /* CUDA runtime error (message has details) */
#define DC_ERR_NOMEM (-3)     /* device or host allocation failed         */
#define DC_ERR_IO (-4)        /* file could not be read or written        */
#define DC_ERR_CAPACITY (-5)  /* output buffer too small / bound exceeded */
#define DC_ERR_TIMEOUT (-6)   /* a bounded device-side wait ran out       */
#define DC_ERR_NOT_FOUND (-7) /* delete of an edge that is not present    */
#define DC_ERR_STATE (-8)     /* call order (e.g. no decomposition yet)   */
#define DC_ERR_NO_DEVICE (-9) /* no CUDA device / extension unusable      */

/* Message of the calling thread's last failed call ("" if none). */
const char* dc_last_error(void);
/* Library version string. */
const char* dc_version(void);

/* ---- seeded generators (host only, no GPU needed) ----------------------- */

/* Directed Erdos-Renyi G(n, m): m distinct edges (u, v), u != v, uniform,
 * written sorted by (src, dst).  Replaces generateGraph
 * (src/graph_gen.cpp:9-34), which is seeded by time and so not reproducible. */
int dc_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t* src, uint32_t* dst);

/* R-MAT graph with 2^scale vertices and edge_factor * 2^scale draws,
 * quadrant probabilities (a, b, c, 1-a-b-c); self-loops dropped, duplicates
 * removed, labels permuted by a seeded shuffle when permute != 0.  Writes the
 * final edge count to *n_edges; with src or dst NULL it only reports the
 * count.  capacity = length of src/dst.  No reference counterpart (the
 * reference has only the ER generator). */
int dc_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                uint64_t seed, int permute, uint64_t capacity,
                uint32_t* src, uint32_t* dst, uint64_t* n_edges);


/* Update stream over a sorted, duplicate-free edge list: n_ops operations,
 * each an insertion of a uniformly random absent edge (u != v) with
 * probability insert_frac, else a deletion of a uniformly random present
 * edge; generated by applying each operation to a host copy of the edge set,
 * so the stream is valid in sequence.  out_del[i] = 1 marks a deletion.
 * Replaces getRandomInsertEdge / getRandomDeleteEdge (src/graph.cpp:327-380). */
int dc_gen_updates(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, uint64_t n_ops,
                   double insert_frac, uint64_t seed, uint32_t* out_u, uint32_t* out_v, uint8_t* out_del);
/* dc_gen_updates with hot operations: where op_hot[i] = 1, operation i has
 * its source among hot[0..n_hot) (an insertion draws the source from them,
 * a deletion picks a present edge leaving one of them).  Used for streams
 * whose batches concentrate on the highest out-degree vertices. */
int dc_gen_updates_hot(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, uint64_t n_ops,
                       double insert_frac, uint64_t seed, const uint32_t* hot, uint32_t n_hot, const uint8_t* op_hot,
                       uint32_t* out_u, uint32_t* out_v, uint8_t* out_del);

/* ---- file formats (host only, no GPU needed) ---------------------------- */

/* Text graph: "# V" header, then "s t" lines.  Self-loops dropped, duplicate
 * edges kept; prune != 0 removes vertices without edges and renumbers the
 * rest in increasing id order.  Replaces Graph::readFile and
 * pruneEmptyVertices (src/graph.cpp:146-250, 110-144).  With src or dst NULL
 * only *V and *E are reported. */
int dc_text_read_edges(const char* path, int prune, uint32_t* V, uint64_t* E,
                       uint32_t* src, uint32_t* dst, uint64_t capacity);

/* Binary graph "<file>-binary-g=<GAP>" (Graph::readBinary,
 * src/graph.cpp:287-325): the out-lists as an edge list, src ascending. */
int dc_binary_read_edges(const char* path, uint32_t* V, uint64_t* E,
                         uint32_t* src, uint32_t* dst, uint64_t capacity);
/* Graph::writeBinary (src/graph.cpp:261-285) of an edge list, lists in
 * ascending neighbour order, `gap` free slots per list (filled 0xCDCDCDCD). */
int dc_binary_write_edges(const char* path, uint32_t V, uint64_t E,
                          const uint32_t* src, const uint32_t* dst, uint32_t gap);

/* .decomp file (writeDecompFile / readDecompFile, src/utils.h:76-109):
 * kmax, lmax, kmaxes[V], rows[(kmax+1) * V], all int32. */
int dc_decomp_file_write(const char* path, uint32_t V, int32_t kmax, int32_t lmax,
                         const int32_t* kmaxes, const int32_t* rows);
/* Reads the header (and, when kmaxes/rows are given and rows_cap is large
 * enough, the arrays).  V must be the graph's vertex count. */
int dc_decomp_file_read(const char* path, uint32_t V, int32_t* kmax, int32_t* lmax,
                        int32_t* kmaxes, int32_t* rows, uint64_t rows_cap);
/* .decompCPU text file (writeDecompFileCPU, src/utils.h:110-124). */
int dc_decomp_cpu_file_write(const char* path, uint32_t V, const int32_t* kmaxes,
                             const int32_t* rows);

/* ---- device-resident graphs ---------------------------------------------- */

typedef struct dc_graph dc_graph;

typedef struct dc_graph_opts {
    uint32_t gap_min; /* free slots per adjacency list (reference OFFSET_GAP = 1) */
    uint32_t gap_div; /* extra free slots = degree / gap_div (0: none)             */
    int32_t device;   /* CUDA device ordinal, -1 = current device                  */
} dc_graph_opts;

void dc_graph_opts_default(dc_graph_opts* opts);
/* Number of visible CUDA devices (0 when none; never fails). */
int dc_device_count(int* n);
/* Grows the device's stream-ordered memory pool -- the engine allocates all
 * device memory from it and keeps freed blocks there -- to hold at least
 * `bytes`: allocations inside later calls (a store rebuild, a larger
 * skyline) then reuse that memory instead of mapping new pages into the
 * pool, which costs up to hundreds of ms per call for tens of GB.  The memory
 * stays reserved for the process.  No counterpart in the reference (it
 * allocates with cudaMalloc per call, src/cuda_memory.h:5-93). */
int dc_reserve_device_memory(int device, uint64_t bytes);

/* Builds the device CSR (out) + CSC (in) from host edge arrays; the copy to
 * the device is part of the call.  Replaces Graph construction plus
 * allocateDeviceGraphMemory / moveGraphToDevice (src/cuda_memory.h:5-41). */
int dc_graph_create(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                    const dc_graph_opts* opts, dc_graph** out);
/* Same from device-resident edge arrays (no host copy). */
int dc_graph_create_device(uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst,
                           const dc_graph_opts* opts, dc_graph** out);
/* Graph(const string&) (src/graph.cpp:381-395): reads "<path>-binary-g=<gap>"
 * when present (or `path` itself when it names such a file), else parses the
 * text file (prune as in dc_text_read_edges). */
int dc_graph_load(const char* path, int prune, const dc_graph_opts* opts, dc_graph** out);
/* Graph::readFile (src/graph.cpp:146-250) with the parse on the GPU: the
 * file's bytes are copied to the device once and split into lines, parsed,
 * compacted and (prune != 0) pruned and renumbered there, then built into
 * the device CSR/CSC.  Same graph, same errors as dc_text_read_edges +
 * dc_graph_create (lines of at most 511 bytes). */
int dc_graph_load_text_device(const char* path, int prune, const dc_graph_opts* opts, dc_graph** out);
int dc_graph_free(dc_graph* g);
int dc_graph_info(const dc_graph* g, uint32_t* V, uint64_t* E);
/* Live in/out degrees (host arrays of V). */
int dc_graph_degrees(dc_graph* g, int32_t* in_deg, int32_t* out_deg);
/* Live edges, src ascending, dst ascending within a source.  With src/dst
 * NULL only *n_edges is reported. */
int dc_graph_get_edges(dc_graph* g, uint32_t* src, uint32_t* dst, uint64_t capacity, uint64_t* n_edges);
/* Graph::writeBinary of the current device graph. */
int dc_graph_write_binary(dc_graph* g, const char* path, uint32_t gap);
/* Device bytes the handle holds now (adjacency with slack, decomposition,
 * engine scratch).  No counterpart in the reference; the serving loop charges
 * it against its HBM budget. */
int dc_graph_device_bytes(const dc_graph* g, uint64_t* bytes);

/* ---- decomposition ------------------------------------------------------- */

#define DC_METHOD_INCREMENTAL 0 /* kmax + row 0 by peeling, rows 1..kmax derived row to row */
#define DC_METHOD_PEEL 1        /* one fresh peel per row, the reference's schedule          */

/* dcore(Graph&) (main.cu:197-262), also checkDCore (main.cu:276-293): kmax of
 * every vertex and all rows lmax[k][v], k = 0..kmax, kept on the device.
 * Reports the global kmax and lmax.  Both methods give identical results. */
int dc_decompose(dc_graph* g, int method, int32_t* kmax, int32_t* lmax);
/* A slice of the decomposition, for sharding rows over GPUs that each hold
 * the whole graph (each row k depends only on the graph and on kmax): kmax
 * and row 0 (computed when k_first = 0 or when not current), then rows
 * max(k_first, 1)..k_last only, clamped to kmax (an empty range: kmax and
 * row 0 alone).  Rows of the
 * range are derived from row 0 directly, so ranges are independent.
 * Afterwards row 0 and the range can be read (dc_get_lmax_rows); reading
 * other rows, the skyline or writing files fails with DC_ERR_STATE until a
 * full dc_decompose.  No reference counterpart (dcore computes all rows,
 * main.cu:236-243). */
int dc_decompose_rows(dc_graph* g, uint32_t k_first, uint32_t k_last, int32_t* kmax, int32_t* lmax);
/* Work weights for row sharding: weights[k] = total in + out degree of the
 * vertices with kmax >= k (k = 0..kmax; capacity >= kmax + 1).  Needs kmax
 * (dc_decompose or dc_decompose_rows). */
int dc_row_weights(dc_graph* g, uint64_t* weights, uint64_t capacity);

typedef struct dc_decomp_info {
    int32_t kmax, lmax;
    uint64_t n_corners; /* skyline corners stored on the device */
    float kmax_ms, row0_ms, rows_ms, skyline_ms, expand_ms;
    uint64_t evals, drops; /* row-to-row evaluations and value drops */
    uint64_t entries;      /* adjacency entries read by the row-to-row kernel */
} dc_decomp_info;
int dc_decomp_info_get(dc_graph* g, dc_decomp_info* info);

/* g.kmaxes (host array of V). */
int dc_get_kmaxes(dc_graph* g, int32_t* out);
/* Rows k0..k0+n-1 of g.lmaxes, row-major, V values per row, into host memory
 * (pinned memory from dc_host_alloc gives full copy bandwidth). */
int dc_get_lmax_rows(dc_graph* g, uint32_t k0, uint32_t n, int32_t* out);
/* Same into device memory. */
int dc_get_lmax_rows_device(dc_graph* g, uint32_t k0, uint32_t n, int32_t* d_out);
/* Keeps all (kmax+1) * V rows dense on the device (later row reads are copies). */
int dc_materialize_rows(dc_graph* g);
int dc_release_rows(dc_graph* g);
/* Compact skyline: off[V+1]; corners off[v]..off[v+1]-1 of v as (k, l) pairs
 * with k ascending; lmax[k][v] = l of the last corner with k_i <= k for
 * k <= kmax[v], 0 above.  With off/ks/ls NULL only *n_corners is reported. */
int dc_get_skyline(dc_graph* g, uint32_t* off, int32_t* ks, int32_t* ls, uint64_t capacity,
                   uint64_t* n_corners);
/* writeDecompFile / writeDecompFileCPU of the current decomposition. */
int dc_write_decomp(dc_graph* g, const char* path);
int dc_write_decomp_cpu(dc_graph* g, const char* path);
/* writeDecompFileCPU (src/utils.h:110-124) with the text formatted on the
 * GPU from the device skyline and copied to the host once; byte-identical to
 * dc_write_decomp_cpu. */
int dc_write_decomp_cpu_device(dc_graph* g, const char* path);

/* ---- maintenance ------------------------------------------------------- */

#define DC_MAINT_AUTO 0   /* the engine's scheduler picks per batch            */
#define DC_MAINT_LOCAL 1  /* kmax and row 0 updated locally (h-index refine)   */
#define DC_MAINT_REPEEL 2 /* kmax and row 0 recomputed by the fused full peel  */

typedef struct dc_maint_stats {
    uint64_t inserted, deleted; /* net edge insertions / deletions applied            */
    int32_t kmax, lmax;         /* after the batch                                    */
    int32_t rows_recomputed;    /* rows 0..R recomputed (R + 1); rows above kept      */
    int32_t method;             /* DC_MAINT_LOCAL or DC_MAINT_REPEEL                  */
    uint32_t rebuilt;           /* 1 when the adjacency store grew (slack exhausted)  */
    uint32_t rows_local;        /* rows repaired in place: bit 0 deletions, bit 1 insertions */
    uint64_t region;            /* vertices visited by the local kmax / row-0 update  */
    float apply_ms, core_ms, rows_ms, total_ms;
    float del_repair_ms;        /* in-place row repair of the deletions (0: none ran) */
    float ins_repair_ms;        /* in-place row repair of the insertions (0: none ran) */
    uint64_t ins_scanned;       /* list entries the insertion repair read             */
    uint32_t captured;          /* 1 when the batch ran as one captured CUDA graph    */
    uint32_t reserved;
} dc_maint_stats;

/* maintenanceFast (main.cu:1665-1751) / maintenance (main.cu:1536-1663):
 * applies a batch of b edge updates to the device graph and brings the
 * decomposition up to date.  pairs[2*i], pairs[2*i+1] = (from, to);
 * is_delete[i] != 0 marks a deletion (is_delete NULL: all insertions).  The
 * batch has sequential semantics and is applied as its net effect per edge;
 * deleting an edge that is not present fails with DC_ERR_NOT_FOUND and leaves
 * the graph unchanged.  Afterwards kmaxes and every row equal a full
 * decomposition of the updated graph.  A graph without a decomposition is
 * decomposed first.  stats may be NULL. */
int dc_maintain(dc_graph* g, const uint32_t* pairs, const uint8_t* is_delete, uint64_t b, int method,
                dc_maint_stats* stats);
/* Row maintenance mode (default 1).  Repair: the deletions of a batch are
 * applied first and rows 1..R are repaired in place from their old values,
 * touching only the vertices the deletions reach; the insertions follow as a
 * second batch whose rows are repaired in place row after row (values can
 * only rise: a region grown from the inserted edges and the vertices that
 * joined C_k, bounded by the new previous row, refined down to the new row).
 * A repair falls back to recomputing rows 1..R from the new row 0 when a
 * row's region outgrows a block's table or when it has run as long as that
 * recomputation is expected to take (the rows phase of the last full
 * decomposition scaled by R / kmax).  1: repair when the batch has at most
 * 64 net updates and the lists they touch are short enough that the repair
 * is expected to beat recomputation; 2: repair whenever the updates fit, with no time
 * limit; 3: repair whenever the updates fit, within the time limit (the
 * learned scheduler's incremental path); 0: every batch recomputes rows 1..R
 * from the new row 0.  Results are identical.  The
 * reference re-peels rows k <= M+1 (main.cu:1735-1743); its disabled exact
 * l-list maintenance (kListFindUpperBound / kListRefineHIndex, main.cu:929-1242,
 * hInIndex src/cuda_utils.cuh:68-77) is the specification this replaces. */
int dc_set_row_repair(dc_graph* g, int on);
/* Captured batches (default 1): a batch of one kind of update (deletions or
 * insertions, after its net effect) on the local method with rows repaired
 * in place (row mode 1 and at most 64 net updates, or modes 2 and 3 and at
 * most 1536) runs as ONE CUDA graph launch -- upload, checks, list updates,
 * kmax / row-0 update, row bound, row repair, skyline merge and the status
 * read-back -- with every branch between its kernels taken on the device.
 * A batch whose lists lack free slots, whose repair is not expected to pay
 * or gives up, or whose merged skyline outgrows its buffer is finished on
 * the host from the state the graph left (dc_maint_stats.captured tells
 * which ran).  A mixed batch split into deletions and insertions (row
 * repair) runs as two graphs.  0 keeps every batch host-driven.  Results are
 * identical.  No counterpart in the reference (a host loop drives every
 * kernel and polls the device between them, main.cu:741-746, 1735-1743). */
int dc_set_captured_batches(dc_graph* g, int on);

/* ---- learned maintenance scheduler -------------------------------------- */
/* A BF16 MLP (16 -> 64 -> 64 -> 2, ReLU) predicting the log of the time of
 * a batch on each of two paths from 16 features of the batch
 * (dc_maint_log_get lists them): output 0 the incremental path
 * (DC_MAINT_LOCAL with rows repaired in place wherever the batch fits, mode 3
 * of dc_set_row_repair), output 1 the full path (DC_MAINT_REPEEL with rows
 * 1..R recomputed, mode 0).  DC_MAINT_AUTO runs the path with the smaller
 * prediction for batches of at most 65,536 net updates (larger ones always
 * take the full path); with no network attached the rule of thumb decides
 * (at most 64 net updates: local; rows by the graph's row mode).  Both paths
 * give exact results.  Training and inference run in the engine's own CUDA
 * kernels.  No reference counterpart (the reference fixes its batching mode
 * at compile time, src/common.h:18-19, and always re-peels rows,
 * main.cu:1735-1743). */
typedef struct dc_sched dc_sched;
int dc_sched_create(uint64_t seed, dc_sched** out);
int dc_sched_free(dc_sched* s);
int dc_sched_param_count(void);
/* fp32 parameters, layout W1[64][16], b1[64], W2[64][64], b2[64], W3[2][64], b3[2] */
int dc_sched_get_params(dc_sched* s, float* params);
int dc_sched_set_params(dc_sched* s, const float* params);
/* input normalisation x' = (x - mean) * scale, 16 values each */
int dc_sched_set_norm(dc_sched* s, const float* mean, const float* scale);
/* Y[n][2] = network(X[n][16]) */
int dc_sched_predict(dc_sched* s, const float* X, uint64_t n, float* Y);
/* Gradient (fp32, dc_sched_param_count values) and loss of the mean squared
 * error over the (sample, output) pairs with M != 0; parameters unchanged. */
int dc_sched_grad(dc_sched* s, const float* X, const float* T, const uint8_t* M, uint64_t n, float* grad, float* loss);
/* `epochs` full-batch Adam steps on the same loss. */
int dc_sched_train(dc_sched* s, const float* X, const float* T, const uint8_t* M, uint64_t n, int epochs, float lr,
                   float* final_loss);
/* Attach (or with NULL detach) a scheduler to a graph for DC_MAINT_AUTO. */
int dc_graph_set_scheduler(dc_graph* g, dc_sched* s);
/* Feature / timing log of maintained batches (training data). */
int dc_maint_log_enable(dc_graph* g, int on);
int dc_maint_log_get(dc_graph* g, float* features, int32_t* methods, float* times_ms, uint64_t capacity, uint64_t* n);

/* getKmaxEdgeBatches with KEDGE_BATCHING (main.cu:1441-1488): partitions an
 * insert batch into sub-batches whose roots (endpoint with the larger kmax,
 * target on ties) share one kmax and are pairwise distinct, buckets in
 * ascending kmax, edges in input order.  batch_of[e] = sub-batch of edge e
 * (numbered as the reference appends them); *n_batches = their number.
 * Host only. */
int dc_kmax_edge_batches(uint32_t V, const int32_t* kmaxes, uint64_t B, const uint32_t* from, const uint32_t* to,
                         int64_t* batch_of, int64_t* n_batches);

/* The same partition on the GPU, for batches already in device memory:
 * d_from[B], d_to[B] (device) against the graph's current kmax values (after
 * dc_decompose or dc_maintain), d_batch_of[B] (device) receives the
 * sub-batch of every edge, numbered exactly as dc_kmax_edge_batches numbers
 * them; *n_batches (host) their number.  Runs on the graph's stream with
 * O(B) work and scratch (a stable radix sort of the edges by root), where the
 * reference allocates and scans a vector<bool>(V) per sub-batch on the host
 * (getKmaxEdgeBatches, main.cu:1441-1488; vector<bool> at main.cu:1469).
 * B < 2^31. */
int dc_graph_kmax_edge_batches(dc_graph* g, uint64_t B, const uint32_t* d_from, const uint32_t* d_to,
                               int64_t* d_batch_of, int64_t* n_batches);

/* kmax of every vertex (in-degree core numbers, the values dc_decompose
 * reports through dc_get_kmaxes) without allocating any device memory.  No
 * counterpart in the reference: it is for callers that cannot let a library
 * call cudaMalloc -- code that owns all device memory through its own pool,
 * or serving loops where cudaMalloc's device-wide synchronisation would stall
 * other work.  The graph comes as plain device arrays: in_off[V+1] (CSC
 * offsets; in-degree of v = in_off[v+1] - in_off[v]), out_off[V+1] and
 * out_nbr[E] (CSR), with out_off[0] = in_off[0] = 0 and out_off[V] =
 * in_off[V] = E (checked: DC_ERR_INVALID otherwise).  kmax[V] is written on
 * the device, the largest value to *kmax_max (may be NULL); the call waits
 * for the GPU before returning.
 * Limits: V <= 262,144 and E <= 4,194,304 (DC_ERR_CAPACITY beyond).  All
 * intermediate state lives in one fixed device array of about 11 MB that
 * this library reserves on every GPU that loads it, until process exit; all
 * calls share it, so calls that overlap on the GPU race and must be
 * serialised by the caller.  The first call on each device looks up that
 * array's address (cudaGetSymbolAddress) and should come before any stream
 * capture on that device.  stream is a cudaStream_t (NULL: default stream). */
int dc_kmax_noalloc(uint32_t V, uint64_t E, const uint32_t* d_in_off, const uint32_t* d_out_off,
                    const uint32_t* d_out_nbr, int32_t* d_kmax, int32_t* kmax_max, void* stream);

/* ---- serving loop ------------------------------------------------------ */
/* Many device-resident graphs, each receiving a stream of edge-update
 * requests.  No counterpart in the reference (its driver, main.cu:1784-2218,
 * loads one graph and runs one operation).  max_concurrent worker threads each
 * take the graph with the oldest pending request, coalesce ALL of that
 * graph's pending requests into one dc_maintain batch (continuous batching;
 * the result equals applying them one by one in submission order) and run it
 * on the graph's own stream, so batches of different graphs overlap on the
 * GPU.  A graph is built and decomposed on the device when first needed; the
 * each resident graph is charged an upper bound of its device footprint
 * (maintenance transients included, room for E/8 more edges), and the
 * charges are kept within hbm_budget_bytes by evicting the least recently
 * used idle graph (its edges move to host memory; it is rebuilt on its next
 * request).  A graph larger than the whole budget is admitted alone; a batch
 * that outgrows its charge while every other resident graph is busy runs
 * over budget.  Reading rows back (dc_server_graph_result) stages up to
 * 2 x min(256 MB, rows) outside the budget.  method: DC_MAINT_*. */
typedef struct dc_server dc_server;
typedef struct dc_server_info {
    uint64_t budget_bytes, used_bytes, peak_bytes;
    uint64_t admissions, evictions, batches, submitted, completed;
    uint64_t measured_bytes; /* dc_graph_device_bytes summed over resident graphs */
    uint32_t graphs, resident;
} dc_server_info;
int dc_server_create(uint64_t hbm_budget_bytes, int max_concurrent, int method, int device, dc_server** out);
/* Registers a graph (copied to host memory; built on the device on demand). */
int dc_server_add_graph(dc_server* s, uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                        uint32_t* graph_id);
/* Queues b updates (pairs[2i], pairs[2i+1]; is_delete may be NULL = all
 * inserts); returns at once.  *request_id numbers requests from 1. */
int dc_server_submit(dc_server* s, uint32_t graph_id, const uint32_t* pairs, const uint8_t* is_delete, uint64_t b,
                     uint64_t* request_id);
/* Waits until every submitted request has completed (DC_ERR_TIMEOUT after
 * timeout_ms). */
int dc_server_drain(dc_server* s, uint64_t timeout_ms);
/* Completed requests since the last call, in completion order: id, graph,
 * latency (submission to end of its batch), requests and updates in its
 * batch, status.  With ids NULL only *n (the number waiting) is reported. */
int dc_server_completions(dc_server* s, uint64_t* ids, uint32_t* graphs, double* latency_ms,
                          uint32_t* batch_requests, uint64_t* batch_updates, int32_t* status, uint64_t capacity,
                          uint64_t* n);
int dc_server_info_get(dc_server* s, dc_server_info* info);
/* Decomposition of one graph after all its queued requests: kmax[V] and,
 * when rows is not NULL, dense rows 0..kmax (rows_capacity >= (kmax+1)*V). */
int dc_server_graph_result(dc_server* s, uint32_t graph_id, int32_t* kmaxes, int32_t* rows, uint64_t rows_capacity,
                           int32_t* kmax);
int dc_server_free(dc_server* s);
/* Row maintenance mode (dc_set_row_repair) of the graphs this server builds
 * from now on (default 1). */
int dc_server_set_row_repair(dc_server* s, int on);

/* ---- diagnostics ------------------------------------------------------- */
/* Per-step timing of the persistent kernels: after each kernel, fn is called
 * with its phase name and `steps` records of 8 words (%globaltimer ns at step
 * start, when the step's work ran out, queue items of the step,
 * %globaltimer at the closing barrier, latest block wake-up, latest block
 * seeding done, earliest block wake-up, unused).  max_steps = 0 turns
 * tracing off. */
typedef void (*dc_trace_fn)(const char* phase, const unsigned long long* rec, unsigned steps, void* user);
int dc_set_trace(dc_graph* g, uint32_t max_steps, dc_trace_fn fn, void* user);
/* Persistent-kernel blocks per SM for every persistent kernel (0 = the
 * default, 2; dc_set_tuning sets the peel and row kernels separately). */
int dc_set_launch(dc_graph* g, int blocks_per_sm);

/* Launch shapes of the persistent kernels: blocks per SM of the fused peel
 * and of the row kernel, and adjacency entries per peel work item.  No
 * counterpart in the reference (its launches are fixed at <<<256, 1024>>>,
 * src/common.h:32-33).  Any setting gives identical results. */
typedef struct dc_tuning {
    int32_t peel_blocks_per_sm; /* 1..8 (capped by occupancy) */
    int32_t rows_blocks_per_sm; /* 1..8 (capped by occupancy) */
    int32_t peel_chunk;         /* power of two, 16..4096 */
    /* Row segments of a full decomposition: each nonzero s cuts rows 1..kmax
     * after row kmax*s/1000, and the segments run as concurrent launches
     * (each one after the first starts from row 0 inside its first row's
     * core).  Nonzero entries are strictly ascending in 1..999 and precede
     * the zeros; all zero = one launch.  Segments share the SMs: each gets
     * at most 1/n of the row kernel's resident blocks. */
    int32_t rows_split_permille[7];
} dc_tuning;
int dc_get_tuning(dc_graph* g, dc_tuning* t);
int dc_set_tuning(dc_graph* g, const dc_tuning* t);
/* Autotuner: times the decomposition of this graph under candidate launch
 * shapes (peel grid 1..6 blocks per SM x chunk 32..256 on the peel alone,
 * then the row kernel's grid 1..8 blocks per SM on the rows alone, each
 * candidate twice, grids capped by occupancy), then row segments: the
 * cumulative cost of rows 1..s is measured at cuts of 5..90 % of kmax (in
 * steps of 5 %), and for one to three cuts the set that balances the
 * segments best is timed (three times); keeps the fastest on the handle and ends with a
 * full decomposition.  *best / *best_ms (may be NULL): the chosen setting and
 * its peel + rows device time. */
int dc_autotune(dc_graph* g, dc_tuning* best, float* best_ms);
/* Row cuts that balance a run of rows over concurrent segments (host only;
 * the autotuner's planner).  cost[i] = measured cost of rows 1..s_i, s_i =
 * kmax * grid[i] / 1000 (grid strictly ascending in 1..999, n in 1..4096);
 * total = cost of all rows.  A segment from cut a to cut b costs about
 * cost[b] - cost[a] (the last one total - cost[last]).  Writes the ncut
 * (1..7, at most n) grid values whose largest segment cost is smallest,
 * ascending, to cuts[0..ncut); *longest (may be NULL) receives that cost. */
int dc_plan_row_cuts(const int32_t* grid, const float* cost, int32_t n, float total, int32_t ncut, int32_t* cuts,
                     float* longest);

/* Limit of every bounded device-side wait of this handle's kernels (grid
 * barriers, work-queue waits), in ns: 0 restores the default of 4 s, else
 * 1 ms .. 600 s.  A wait that runs out ends the kernel and the call returns
 * DC_ERR_TIMEOUT; the handle stays usable.  No reference counterpart (the
 * reference's kernels have no bounded waits and trap on a full buffer,
 * src/cuda_utils.cuh:7,11). */
int dc_set_wait_limit(dc_graph* g, uint64_t ns);
/* Failure-detection tests: block `block` of the handle's next persistent
 * launch leaves at its first grid barrier without arriving, so the other
 * blocks' barrier waits run out and the call returns DC_ERR_TIMEOUT after
 * the wait limit; applies to one launch, -1 cancels.  No reference
 * counterpart. */
int dc_test_withhold_barrier(dc_graph* g, int32_t block);

/* Engine kernel launches since the library was loaded. */
int dc_launch_count(unsigned long long* n);

/* ---- utilities ----------------------------------------------------------- */
int dc_host_alloc(uint64_t bytes, void** p); /* pinned host memory */
int dc_host_free(void* p);
int dc_synchronize(dc_graph* g);
/* The graph's CUDA stream (cudaStream_t) for interop. */
int dc_graph_stream(dc_graph* g, void** stream);

#ifdef __cplusplus
}
#endif

#endif /* DCORE_B200_H */
