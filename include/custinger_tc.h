/* custinger_tc.h - C ABI of the B200 triangle-counting library (libcustinger_tc.so).
 *
 * This is the boundary below the reference's host entry points:
 *   callDeviceAllTriangles     (include/static_triangle_counting/cct.hpp:15-17,
 *                               src/static_triangle_counting/cct.cu:272-277)
 *   callDeviceAllTrianglesCSR  (tests/cct_csr.cu:279-285, declared tests/cct.cpp:25-28)
 *   callDeviceNewTriangles     (src/streaming_triangle_counting/cct_upd.cu:412-440)
 * and the cuStinger graph handle they take (externals/cuStinger, absent from the reference
 * tree; its use is at tests/cct.cpp:261-277 and tests/cct_upd.cpp:227-244,391-398).
 * The C++ drop-in layer (cuStinger.hpp, static_triangle_counting/cct.hpp,
 * streaming_triangle_counting/cct_upd.hpp) is a thin wrapper over these functions.
 *
 * Plain pointers and sizes only. `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream, like the reference's launches). Every function returns a tc_status;
 * tc_last_error() gives a message for the last failure on the calling thread.
 *
 * Graph requirements (checked): ids in [0, nv), every adjacency list strictly ascending
 * (sorted, no duplicates), no self-loops, symmetric (u in N(v) iff v in N(u)). These are the
 * graphs the reference's readers produce. Asymmetry is detected with a 64-bit signed edge
 * checksum (an asymmetric graph passes with probability about 2^-64).
 *
 * Count conventions (bit-exact against the reference):
 *   TC_PV_HANDLE  per-vertex out[v] = 2 t(v) (int32, wraps mod 2^32), what
 *                 devicecuStingerAllTriangles writes (cct.cu:216-270); sum = 6T.
 *   TC_PV_CSR     per-vertex out[v] = sum over w in N(v), w > v of |N(v) ∩ N(w)|, what
 *                 count_all_trianglesGPU writes (tests/cct_csr.cu:228-276); sum = 3T.
 *   `triangles`   outputs are T, the number of triangles (int64). The reference's CPU
 *                 counter hostCountTriangles reports 6T (tests/cct.cpp:71-89).
 */
#ifndef CUSTINGER_TC_H_
#define CUSTINGER_TC_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int tc_status;
enum {
  TC_OK = 0,
  TC_ERR_INVALID_ARG = 1,   /* bad pointer, size or option */
  TC_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  TC_ERR_OOM = 3,           /* device allocation failed */
  TC_ERR_BAD_GRAPH = 4,     /* unsorted/duplicate list, self-loop or id out of range */
  TC_ERR_NOT_SYMMETRIC = 5, /* adjacency is not symmetric */
  TC_ERR_CAPACITY = 6,      /* input larger than a fixed capacity (captured plans, no-alloc paths) */
  TC_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
  TC_ERR_STATE = 8          /* call out of order (e.g. counting a batch that was not applied) */
};

/* Per-vertex output conventions. TC_PV_HANDLE64 is TC_PV_HANDLE (2 t(v)) into int64 entries,
 * which do not wrap where 2 t(v) passes 2^31 (R-MAT 24 hubs): the per_vertex argument then
 * points to int64_t[nv] (cast to int32_t*). No reference counterpart: its outputs are int32. */
enum { TC_PV_NONE = 0, TC_PV_HANDLE = 1, TC_PV_CSR = 2, TC_PV_HANDLE64 = 3 };

/* Memory space of caller pointers. */
enum { TC_MEM_DEVICE = 0, TC_MEM_HOST = 1 };

/* Scheduler: which intersection strategy each oriented edge uses and the launch shapes.
 * tc_sched_default() fills the fixed degree-threshold heuristic. */
typedef struct tc_sched {
  int32_t warp_max_deg;   /* static count: a centre (the edge endpoint whose N+ is hashed) with
                             out-degree up to this is counted by one warp (<= 128), above by a CTA */
  int32_t search_ratio_x16; /* streaming delta count: edge {x,y} binary-searches the shorter list
                               into the longer one when 16 d_long > ratio * d_short (log2 d_long + 1),
                               else merges */
  int32_t blocks_per_sm;  /* persistent grid = SMs x blocks_per_sm (0 = occupancy limit) */
  int32_t chunk;          /* vertices a warp claims per work-queue grab */
  int32_t use_table;      /* 1 = the per-degree-cell strategy table below overrides the rules */
  uint8_t table[16][16];  /* strategy per cell [log2 d_a][log2 d_b]. Static count (a = the centre's
                             out-degree, b = the other endpoint's): 0 = the warp streams N+(b)
                             through the hash set, 1 = one lane walks it, 2 = packed (see
                             packed_max_deg). Streaming: 0 = search, 1 = merge, 2 = stage (the
                             longer list copied into shared memory in pieces with cp.async, each
                             shorter-list entry binary-searched there) */
  int32_t shard;          /* multi-GPU work split (1 = everything): this call counts shard `shard` of */
  int32_t nshards;        /* `nshards`. Static count: a contiguous range of edge centres, the ranges
                             balanced by each centre's predicted intersection work (every rank
                             computes the same ranges from the same graph). Streaming: the changed
                             edges whose canonical key hashes to `shard` (mod nshards). Per-vertex outputs and totals are
                             then partial sums that add up over the shards. */
  int32_t cell_filter;    /* timing mode for scheduler training: -1 = intersect every edge (normal),
                             -2 = none, c >= 0 = only edges of degree cell c (16*log2 d_a + log2 d_b);
                             counts are partial unless -1 */
  int32_t lane_max_deg;   /* static count rule without a table: lists of at most this many entries
                             are walked by one lane each (several lists per warp step) */
  int32_t packed_max_deg; /* static count rule without a table: lists longer than lane_max_deg and
                             of at most this many entries are packed: the warp walks all such lists
                             of a group of 32 neighbours concatenated, 32 entries per step
                             (0 = never); longer lists are streamed one at a time */
  int32_t stream_hub_min; /* streaming delta count (tc_apply_batch, tc_pipeline): changed edges whose
                             longer-list endpoint holds at least this many of a batch phase's
                             changed edges are counted together at that endpoint, its list hashed
                             once in shared memory (0 = never; every edge on its own) */
} tc_sched;

typedef struct tc_graph tc_graph;

const char* tc_last_error(void);
const char* tc_status_string(tc_status s);
void tc_sched_default(tc_sched* s);

/* Build a graph from a CSR (off: nv+1 int64 offsets, ind: off[nv] int32 ids) in host or
 * device memory. The graph owns a copy in slack-managed device storage: each adjacency list
 * gets capacity for ceil(slack * degree) extra entries (rounded to 16 bytes) for streaming
 * insertions. With validate=1 the graph is checked (requirements above); the call then
 * synchronises `stream`. Replaces initializeCuStinger with eInitStateCSR. */
tc_status tc_graph_create(int32_t nv, const int64_t* off, const int32_t* ind, int mem, double slack,
                          int validate, void* stream, tc_graph** out);
tc_status tc_graph_destroy(tc_graph* g);
/* nv, directed edges in use, directed edge slots allocated. */
tc_status tc_graph_info(const tc_graph* g, int32_t* nv, int64_t* edges_used, int64_t* edges_alloc);
/* Copy the graph back as a compact CSR into host arrays (off: nv+1, ind: edges_used). Syncs. */
tc_status tc_graph_export(tc_graph* g, int64_t* off_host, int32_t* ind_host);
/* Full structural check (sorted, no duplicates, no self-loops, ids in range, symmetric). Syncs. */
tc_status tc_graph_validate(tc_graph* g, void* stream);
/* Device pointers of the live structure: per-vertex list start (int64[nv]), used length
 * (int32[nv]) and the adjacency pool. Valid until the next structural update. */
tc_status tc_graph_device_view(tc_graph* g, const int64_t** start, const int32_t** used, const int32_t** pool);

/* What a count measured, read back to the host on request. */
typedef struct tc_count_info {
  int64_t triangles;         /* T */
  int64_t edges_intersected; /* undirected edges {u,v} with deg(u), deg(v) >= 2 */
  int64_t oriented_work;     /* sum over oriented edges u->v of d+(u) + d+(v) (list elements a
                                merge-based intersection reads) */
  int32_t max_out_degree;    /* max d+ in the degree orientation */
  int32_t status;            /* structural check made during the count: TC_OK,
                                TC_ERR_BAD_GRAPH or TC_ERR_NOT_SYMMETRIC */
  int32_t shard_lo;          /* sharded count (sched->nshards > 1): the centres [shard_lo, shard_hi) */
  int32_t shard_hi;          /* it counted (0, -1 when not sharded); */
  int64_t shard_work;        /* their predicted work and that of all centres (units of 16 probes) */
  int64_t total_work;
} tc_count_info;

/* Static count over a graph handle.
 *   pv_mode:       TC_PV_NONE, TC_PV_HANDLE or TC_PV_CSR
 *   per_vertex:    device int32[nv] (required unless TC_PV_NONE), entries [0, nv) overwritten
 *   triangles_dev: optional device int64 receiving T (stream-ordered, no sync)
 *   info:          optional host struct; when given the call synchronises `stream` and returns
 *                  the structural status found during the count as its own status
 *   sched:         NULL = default heuristic
 * Stream-ordered and allocation-free after the first call on a graph of this size, so it can
 * be captured in a CUDA graph once warmed up (with info == NULL). */
tc_status tc_count_static(tc_graph* g, int pv_mode, int32_t* per_vertex, int64_t* triangles_dev,
                          tc_count_info* info, const tc_sched* sched, void* stream);

/* Stateless static count on a caller CSR in device memory (int32 offsets: the raw-CSR path
 * of the reference; int64 offsets for graphs past 2^31 edges). The structural checks run on
 * the fly; their result is in info->status (or in tc_workspace_status() when info == NULL).
 * Uses a per-device workspace owned by the library (grown on demand, freed at exit); calls
 * on one device must not overlap. */
tc_status tc_count_csr32(int32_t nv, const int32_t* d_off, const int32_t* d_ind, int pv_mode,
                         int32_t* per_vertex, int64_t* triangles_dev, tc_count_info* info,
                         const tc_sched* sched, void* stream);
tc_status tc_count_csr64(int32_t nv, const int64_t* d_off, const int32_t* d_ind, int pv_mode,
                         int32_t* per_vertex, int64_t* triangles_dev, tc_count_info* info,
                         const tc_sched* sched, void* stream);

/* Allocation-free variant of tc_count_csr32 (no counterpart in the reference): same inputs,
 * outputs and conventions, but it never calls cudaMalloc or cudaFree. It is for callers that
 * must not allocate device memory when they count: processes whose device memory is owned by
 * another allocator (a framework's caching pool) or reserved in full at start-up, and
 * latency-sensitive loops, where cudaMalloc and cudaFree can synchronise the device. Its working
 * memory is a fixed array inside this library's device image, sized for at most
 * TC_NOALLOC_MAX_NV vertices and TC_NOALLOC_MAX_EDGES directed edges (about 48.6 MiB, held by
 * every GPU that loads the library until the process exits); larger graphs are rejected with
 * TC_ERR_CAPACITY, and a sharded count (sched->nshards > 1) with TC_ERR_INVALID_ARG. All calls
 * share that array and keep the last call's contents (each call clears what must start at zero),
 * so calls that overlap on the GPU race: issue them on one stream or order them with events. The
 * first call on a device looks up the array's device address with that device current. The edge
 * count d_off[nv] is read back to the host, so the call synchronises `stream` once. */
#define TC_NOALLOC_MAX_NV (1 << 20)
#define TC_NOALLOC_MAX_EDGES (1 << 22)
tc_status tc_count_csr32_noalloc(int32_t nv, const int32_t* d_off, const int32_t* d_ind, int pv_mode,
                                 int32_t* per_vertex, int64_t* triangles_dev, tc_count_info* info,
                                 const tc_sched* sched, void* stream);

/* The multi-GPU split rule of the static count on the host: lo[r] = first centre of shard r of
 * nshards (lo[0] = 0, lo[nshards] = n) given prefix[0..n], the exclusive prefix of the centres'
 * predicted work. The device applies the same rule to its own prefix. */
tc_status tc_shard_ranges(const int64_t* prefix_host, int32_t n, int32_t nshards, int32_t* lo_host);

/* Fault injection for tests (host side, no GPU fault): while bytes > 0, every device allocation
 * the library makes that is larger than `bytes` fails as cudaMalloc fails when memory runs out,
 * so calls return TC_ERR_OOM and leave their objects usable. 0 removes the cap. */
tc_status tc_debug_alloc_cap(int64_t bytes);

/* Read back the info of the last stateless count on the current device. Syncs `stream`. */
tc_status tc_workspace_status(void* stream, tc_count_info* info);
/* Free the working memory the stateless counts (tc_count_csr32/64) keep on the current device
 * (it is allocated again by the next such count). Waits for the device first. */
tc_status tc_workspace_release(void);

/* ---- streaming updates ------------------------------------------------------------------ */

/* What one batch did, read back on request. */
typedef struct tc_batch_info {
  int64_t updates;           /* pairs submitted */
  int64_t inserted;          /* undirected edges inserted */
  int64_t deleted;           /* undirected edges deleted */
  int64_t ignored;           /* self-loops, repeats, inserts of present / deletes of absent edges */
  int64_t triangles_added;   /* triangles created by the insertions */
  int64_t triangles_removed; /* triangles destroyed by the deletions */
  int32_t status;
} tc_batch_info;

/* Apply a batch of b undirected edge updates {src[i], dst[i]} (host or device arrays per `mem`;
 * is_delete[i] != 0 marks a deletion, NULL = all insertions) and count the triangles they
 * create and destroy. Set semantics: an edge is present or absent; repeats, self-loops,
 * insertions of present edges and deletions of absent edges are ignored; within a batch all
 * deletions apply before all insertions.
 *   per_vertex:  optional device int32[nv], accumulated: += 2 (t_after(v) - t_before(v))
 *   delta_dev:   optional device int64, accumulated: += T_after - T_before
 *   info:        optional host struct (the call then synchronises `stream`)
 * The call synchronises once per batch to size list relocations. */
tc_status tc_apply_batch(tc_graph* g, const int32_t* src, const int32_t* dst, const uint8_t* is_delete, int64_t b,
                         int mem, int32_t* per_vertex, int64_t* delta_dev, tc_batch_info* info, const tc_sched* sched,
                         void* stream);

/* The cuStinger batch steps on directed entries in device memory (a batch is expected to be
 * symmetric: both directions of every edge).
 * tc_batch_sort:     sort (src, dst) in place by (src, dst); offsets[nv+1] = batch CSR over src;
 *                    dup[i] = 1 for self-loops and repeats of an earlier entry (sortDeviceBUD).
 * tc_insert_sorted:  insert the entries with dup == 0, flagging (dup = 1) those already present
 *                    (edgeInsertionsSorted); *not_fitting = entries whose list had to move.
 * tc_delete_sorted:  delete the entries with dup == 0 that are present (edgeDeletionsSorted).
 * tc_count_batch:    after an insertion (sign = +1): per_vertex[v] += 2 for each vertex of each
 *                    triangle containing a batch entry with dup == 0 (callDeviceNewTriangles);
 *                    before a deletion (sign = -1): the same for the triangles the deletion
 *                    destroys, subtracted. delta_dev (optional) += sign * triangles. */
tc_status tc_batch_sort(int32_t nv, int32_t* d_src, int32_t* d_dst, int64_t b, int32_t* d_offsets, int32_t* d_dup,
                        void* stream);
tc_status tc_insert_sorted(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, int64_t b, int32_t* d_dup,
                           int64_t* not_fitting, void* stream);
tc_status tc_delete_sorted(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, const int32_t* d_dup, int64_t b,
                           void* stream);
tc_status tc_count_batch(tc_graph* g, const int32_t* d_src, const int32_t* d_dst, const int32_t* d_offsets,
                         const int32_t* d_dup, int64_t b, int sign, int32_t* per_vertex, int64_t* delta_dev,
                         const tc_sched* sched, void* stream);

/* ---- captured streaming pipeline (no counterpart in the reference: its driver launches the
 * three streaming kernels one by one per batch, cct_upd.cu:412-440) ------------------------------
 *
 * The same semantics as tc_apply_batch for device batches, as one CUDA graph launch per batch
 * with no host synchronisation inside it. Batches are binned by size (capacities 2^10, 2^11, ...
 * up to max_batch, until the autotuner merges bins); each bin's graph is captured on first use
 * with launches sized for the bin and reads the batch's counts on the device. The triangle
 * delta of each phase of a batch (deletions, insertions) is one persistent kernel over a
 * resident grid: each warp runs its share of the per-edge pass, then takes the queued chunks of
 * long intersections as other warps publish them (each wait for a chunk is bounded). Pool
 * headroom for the worst case of a batch (every list it touches relocating) is reserved before
 * each launch.
 *
 * tc_pipeline_create: for batches of at most max_batch updates on graph g (the graph must not be
 *                     updated through other calls while the pipeline has a batch in flight).
 * tc_pipeline_apply:  enqueue one batch (device arrays; d_is_delete may be NULL = insertions) on
 *                     `stream`. per_vertex (+= 2 per vertex per triangle created, -= 2 per one
 *                     destroyed; NULL = internal scratch) and delta_dev (+= created - destroyed;
 *                     NULL allowed) are updated when the graph runs. Returns after the launch; the
 *                     previous batch is settled first (its status folded into the graph).
 * tc_pipeline_prepare: reserve pool headroom for max_batch and capture every bin's graph for these
 *                     outputs now (optional; otherwise both happen on first use).
 * tc_pipeline_sync:   wait for the last batch and report it (errors of that batch surface here;
 *                     TC_ERR_TIMEOUT when a delta kernel's wait for queued work ran out).
 * tc_pipeline_autotune: explore over the next `batches` batches: each runs under one arm of its
 *                     natural bin, a candidate tile shape of the delta kernel (CTAs per SM: the
 *                     occupancy limit; split threshold / split-item size 2048/1024, 1024/512,
 *                     512/256, 256/128 or 128/64 entries) or the default shape in the next bin's graph,
 *                     timed with events. Afterwards each bin keeps its fastest shape, and a bin
 *                     whose batches ran at most 3 % slower in the next bin's graph is merged into
 *                     it (its threshold dropped).
 * tc_pipeline_info:   bins, their capacities and the delta-kernel CTAs per SM each uses.
 * tc_pipeline_plan_get / _set: the tuned bins and shapes, to carry a tuning over to another
 *                     pipeline with the same max_batch (e.g. tuned on a copy of the graph).
 * tc_pipeline_profile: record events around the two delta kernels inside the captured graphs
 *                     (drops the graphs when it changes; call before tc_pipeline_prepare) and
 *                     count their algorithmic bytes, sum over changed edges {x,y} of
 *                     4 (deg x + deg y) + 8; tc_pipeline_stats returns the totals since.
 * tc_pipeline_set_wait_bound: the bound of the delta kernels' wait for queued work (default 2 s)
 *                     and a number of warps it waits for beyond the grid (0 normally; a test gives
 *                     1 to make the waits run out and checks that the batch reports
 *                     TC_ERR_TIMEOUT with the device still usable). Drops the captured graphs. */
typedef struct tc_pipeline tc_pipeline;
typedef struct tc_pipeline_plan {
  int32_t nbins;
  int64_t bin_cap[16];     /* bin capacities (the fine ladder) */
  int32_t serve[16];       /* bin whose graph runs the batches of bin i (>= i; > i where merged) */
  int32_t ctas_per_sm[16]; /* delta kernel shape of that graph: CTAs per SM (0 = occupancy limit), */
  int32_t chunk[16];       /* split-item size and */
  int32_t split_min[16];   /* split threshold (entries of the shorter list) */
} tc_pipeline_plan;
tc_status tc_pipeline_create(tc_graph* g, int64_t max_batch, const tc_sched* sched, tc_pipeline** out);
tc_status tc_pipeline_apply(tc_pipeline* p, const int32_t* d_src, const int32_t* d_dst, const uint8_t* d_is_delete,
                            int64_t b, int32_t* per_vertex, int64_t* delta_dev, void* stream);
tc_status tc_pipeline_prepare(tc_pipeline* p, int32_t* per_vertex, int64_t* delta_dev, void* stream);
tc_status tc_pipeline_sync(tc_pipeline* p, tc_batch_info* last);
tc_status tc_pipeline_autotune(tc_pipeline* p, int32_t batches);
tc_status tc_pipeline_info(const tc_pipeline* p, int32_t* nbins, int64_t* bin_cap, int32_t* delta_blocks_per_sm);
tc_status tc_pipeline_plan_get(const tc_pipeline* p, tc_pipeline_plan* plan);
tc_status tc_pipeline_plan_set(tc_pipeline* p, const tc_pipeline_plan* plan);
tc_status tc_pipeline_profile(tc_pipeline* p, int on);
tc_status tc_pipeline_stats(tc_pipeline* p, int64_t* batches, double* delta_ms, int64_t* delta_bytes);
tc_status tc_pipeline_set_wait_bound(tc_pipeline* p, uint64_t wait_ns, int32_t extra_arrivals);
tc_status tc_pipeline_destroy(tc_pipeline* p);

/* Per degree-cell statistics of the oriented edges of the last static count, filed as the count
 * files them: a = the larger out-degree of the two endpoints (the centre's), b = the smaller,
 * cell = 16*min(15, log2 a) + min(15, log2 b). out[4*c + 0..3] = edge count, sum of
 * log2(1 + a), sum of log2(1 + b), sum of b/a. Host array of 1024 doubles. Syncs. */
tc_status tc_cell_stats(tc_graph* g, double* out_host, void* stream);

/* ---- autotuner --------------------------------------------------------------------------- */

/* Time the candidate scheduler settings (out-degree threshold of the warp path, search ratio,
 * work-queue chunk, CTAs per SM) on this graph, `reps` timed runs each after one warm-up, and
 * return the fastest in *best (its median time in *best_ms). The result is also cached under
 * the graph's (log2 n, log2 m, log2 max out-degree) bucket. */
tc_status tc_autotune_static(tc_graph* g, int pv_mode, int32_t* per_vertex, int32_t reps, tc_sched* best,
                             float* best_ms, void* stream);
/* Cached setting for a graph bucket (TC_ERR_STATE and the default heuristic when none). */
tc_status tc_autotune_lookup(int32_t nv, int64_t edges, int32_t max_out_degree, tc_sched* out);
/* Save / load the cache as text (one line per bucket). */
tc_status tc_autotune_save(const char* path);
tc_status tc_autotune_load(const char* path);

/* ---- learned scheduler: a 3-layer FP32 MLP trained and evaluated on the GPU ------------------ */

/* features (log2(1+d_a), log2(1+d_b), d_min/d_max, cell id / 255) -> 64 -> 64 -> one predicted
 * log2 cost (ns per edge) per strategy. Parameters are TC_MLP_PARAMS floats, layout
 * W1[64][4] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]. */
#define TC_MLP_IN 4
#define TC_MLP_HIDDEN 64
#define TC_MLP_OUT 3
#define TC_MLP_PARAMS                                                                                 \
  (TC_MLP_HIDDEN * TC_MLP_IN + TC_MLP_HIDDEN + TC_MLP_HIDDEN * TC_MLP_HIDDEN + TC_MLP_HIDDEN +         \
   TC_MLP_OUT * TC_MLP_HIDDEN + TC_MLP_OUT)

/* Deterministic He-uniform initialisation into a host array of TC_MLP_PARAMS floats. */
tc_status tc_mlp_init(float* params_host, uint64_t seed);
/* y[n][TC_MLP_OUT] = MLP(x[n][TC_MLP_IN]) (device arrays). */
tc_status tc_mlp_forward(const float* d_params, const float* d_x, int32_t n, float* d_y, void* stream);
/* Gradient of the masked MSE mean_i (y_i[strategy_i] - label_i)^2 into d_grad (TC_MLP_PARAMS
 * floats, overwritten) and the loss into d_loss[0]. */
tc_status tc_mlp_backward(const float* d_params, const float* d_x, const int32_t* d_strategy, const float* d_label,
                          int32_t n, float* d_grad, float* d_loss, void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8; step counts from 1). */
tc_status tc_mlp_adam_step(float* d_params, const float* d_grad, float* d_m, float* d_v, int32_t step, float lr,
                           void* stream);
/* Full-batch Adam for `epochs` steps; the final loss goes to *loss_host (optional, syncs). */
tc_status tc_mlp_train(float* d_params, const float* d_x, const int32_t* d_strategy, const float* d_label, int32_t n,
                       int32_t epochs, float lr, float* loss_host, void* stream);

/* Fill a scheduler from a trained MLP (device parameters) whose outputs are predicted log2
 * costs per edge of each strategy: for every degree cell, the choice among the strategies of
 * `kind` (0 = static count: the warp streams the shorter list, one lane walks it, or the warp
 * walks the group's lists packed: table entries 0, 1, 2 = network outputs 0, 1, 2; 1 = streaming
 * delta: search or merge, table entries 0, 1 = outputs 1, 2) goes into s->table and
 * s->use_table = 1. The fixed rule (static: s->lane_max_deg and s->packed_max_deg; streaming:
 * s->search_ratio_x16; on the cell's mean degrees) is the fallback: a cell takes another
 * strategy only when the network predicts it at least 5% cheaper than the rule's. cell_features
 * (host, 256 x TC_MLP_IN floats: mean log2(1 + a), mean log2(1 + b), mean b/a, cell id / 255, as
 * tc_cell_stats files the cells) describe each cell; NULL uses the cells' nominal degrees. */
tc_status tc_sched_learned(const float* d_params, int kind, const float* cell_features, tc_sched* s, void* stream);
/* The decision step of tc_sched_learned alone, on the host (no GPU): costs (host, 256 x TC_MLP_OUT
 * floats) are the network's outputs for the 256 cells. */
tc_status tc_sched_from_costs(int kind, const float* cell_features, const float* costs, tc_sched* s);

/* Phase timing of counts issued by the calling thread: CUDA events recorded on the launching
 * stream around the orientation passes and around the intersection kernel (off by default;
 * recording adds no synchronisation). */
typedef struct tc_phase_times {
  float orient_ms;   /* orientation: out-degree pass, scan, fill */
  float count_ms;    /* the intersection kernel (k_count) */
  int32_t launches;  /* kernels the last count launched */
} tc_phase_times;
tc_status tc_profile_enable(int on);
/* Times of the last profiled count on this thread; waits for its events. */
tc_status tc_profile_last(tc_phase_times* t);

#ifdef __cplusplus
}
#endif
#endif /* CUSTINGER_TC_H_ */
