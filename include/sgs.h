/*
 * sgs.h -- C ABI of the B200-native incremental streaming-graph engine
 * (drop-in for the hot path of C-GpuStreamGraph).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (0 = ok, < 0 = error; sgs_last_error() gives a thread-local message).  No
 * entry point exits the process (the reference exits through
 * GROUTE_CUDA_CHECK -> HandleError, groute/internal/cuda_utils.h:59-65).
 *
 * Mapping to the reference (paths relative to the reference project):
 *   sgs_create / sgs_config       <- Engine ctor + flags
 *                                    (include/framework/framework.cuh:124-140,
 *                                     include/utils/app_skeleton.h:42-100)
 *   sgs_load_csr / sgs_load_edge_list
 *                                 <- Engine::LoadGraph + Context graph load
 *                                    (framework.cuh:310-384,
 *                                     include/utils/graphs/traversal.h:149-170,
 *                                     src/utils/parser.cpp:296-406)
 *   sgs_query_add                 <- Engine::InitGraph(args...) + Engine::Start
 *                                    (framework.cuh:389-439, :549-584) for the
 *                                    AppBase functors of samples/hybrid_{bfs,
 *                                    sssp,cc,pr}
 *   sgs_apply_batch               <- one snapshot of the sample drivers:
 *                                    del_edge + add_edge (SSSP/BFS/CC,
 *                                    framework.cuh:975-1038, :1507-1655) or
 *                                    Cancelation + Compensate (PR,
 *                                    framework.cuh:1110-1301), with the PMA
 *                                    updates of csr_graph.cuh:658-811
 *   sgs_gather                    <- Engine::GatherValue/GatherParent/
 *                                    GatherBuffer (framework.cuh:1657-1679)
 *   sgs_get_query_stats           <- RunningInfo counters
 *                                    (framework/hybrid_policy.h:38-136)
 *   sgs_cache_refresh             <- compute_hot_vertices_* +
 *                                    confirm_candidate_batch + LoadCache
 *                                    (framework.cuh:149-308, :1304-1385;
 *                                    variants/driver.cuh:437-516); the same
 *                                    admission also runs inside every
 *                                    sgs_apply_batch
 */
#ifndef SGS_H
#define SGS_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SGS_API __attribute__((visibility("default")))
#else
#define SGS_API
#endif

/* status codes */
#define SGS_OK 0
#define SGS_ERR_INVALID (-1)   /* bad argument / out-of-range vertex id   */
#define SGS_ERR_CUDA (-2)      /* CUDA runtime error                       */
#define SGS_ERR_OOM (-3)       /* device or pinned-host allocation failed  */
#define SGS_ERR_STATE (-4)     /* call out of order (e.g. no graph loaded) */
#define SGS_ERR_NOCONV (-5)    /* round limit reached before convergence   */

/* algorithms: the four sample apps */
#define SGS_BFS 0  /* samples/hybrid_bfs  : depth from source             */
#define SGS_SSSP 1 /* samples/hybrid_sssp : integer-weight distance       */
#define SGS_CC 2   /* samples/hybrid_cc   : min id reaching v (directed)  */
#define SGS_PR 3   /* samples/hybrid_pr   : unnormalised delta PageRank   */

/* where caller buffers live */
#define SGS_MEM_HOST 0
#define SGS_MEM_DEVICE 1

/* edge weights (reference: push_functor.h:306 synthesizes (u+v)%128+1) */
#define SGS_W_EXPLICIT 0 /* weights stored per edge (>= 1)                */
#define SGS_W_SYNTH 1    /* (src+dst)%128+1 computed per edge, not stored */
#define SGS_W_UNIT 2     /* every weight 1, not stored                    */

/* gather fields */
#define SGS_FIELD_VALUE 0  /* u32 value (BFS/SSSP/CC); f64 rank (PR)        */
#define SGS_FIELD_PARENT 1 /* u32 parent (BFS/SSSP/CC)                      */
#define SGS_FIELD_BUFFER 2 /* u32 buffer (== value once converged); f64
                              residual (PR)                                 */

typedef struct sgs_engine sgs_engine;

typedef struct sgs_config {
  int device;             /* CUDA device ordinal                           */
  uint32_t segments;      /* -SEGMENT: vertex segments (residency unit)    */
  uint32_t n_stream;      /* -n_stream: accepted for drop-in; unused       */
  uint32_t block_size;    /* -block_size: accepted for drop-in; unused     */
  double cache_gb;        /* -cache: HBM bytes (1e9) of the device edge
                             cache of the host tier, carved out of
                             hbm_budget_gb (needs a budget; 0: no cache).
                             Lines of 128 slots of host-resident blocks are
                             admitted per snapshot by hotness (activations
                             over a four-snapshot window) and copied on a
                             side stream; the static HBM segments get
                             hbm_budget_gb - cache_gb                      */
  double hbm_budget_gb;   /* HBM budget for edge blocks; <= 0: unlimited.
                             Segments beyond it live in pinned host memory
                             and are read over the host link              */
  int weight_mode;        /* SGS_W_*                                        */
  uint32_t max_rounds;    /* round limit per convergence (reference: 1000) */
  double pr_alpha;        /* damping, 0.85 (hybrid_pr_common.h:39)         */
  double pr_tol;          /* stop when sum|residual| < pr_tol              */
  uint32_t slack_div;     /* per-block slack: cap = deg + deg/slack_div + 2 */
  double arena_headroom;  /* extra arena fraction for relocated blocks    */
  uint32_t group_size;    /* BFS/SSSP/CC queries relaxed together per edge
                             pass: 1..4 (narrow groups: lanes in one 32-B
                             sector) or 5..64 (wide groups: one 512-B row
                             per vertex, a warp's threads over the lanes) */
  uint32_t persistent;    /* bit 0: relaxation phases, bit 1: invalidation
                             phases run as one cooperative launch looping
                             over rounds with a grid barrier between them
                             (no host read per batch of rounds); a clear bit:
                             rounds launched in batches with one counter
                             read per batch.  Bit 2 (with bit 0 clear): a
                             narrow group's relaxation phase runs round 0 --
                             a snapshot's sweep -- as a plain launch on the
                             large grid and its later rounds as one
                             cooperative launch.  Bit 3: PageRank's pull
                             rounds (absorb + sweep + convergence test) as
                             one cooperative launch.  Default 14          */
  uint32_t pull;          /* bit 0 (default on): PageRank's all-vertex
                             sweeps as pulls over an in-edge (CSC) store
                             kept in HBM (built by transposing the graph
                             when first needed, then updated by every
                             snapshot); bit 1: BFS-only starts of a narrow
                             group run direction-optimizing (bottom-up
                             rounds over the same store when the frontier
                             is large); 0: push only                      */
  uint32_t host_policy;   /* reads of the host tier during a snapshot's
                             repair (-hybrid): 0 zero-copy (default); 1 the
                             used host arena copied to HBM by the copy
                             engine before every repair; 2 that copy only
                             when the repair's first frontier covers more
                             than half of the slots                        */
  uint32_t pr_warm;       /* 1 (default): a removed PageRank query leaves its
                             vector behind and the next PageRank start
                             continues from it (its residual on the current
                             graph computed first; same tolerance, fewer
                             rounds after small changes); 0: every start
                             from scratch                                  */
  uint32_t repair;        /* bit 0: narrow groups repair after deletions by
                             pulling over the in-edges of the vertices the
                             invalidation reset (in-edge store with
                             weights), instead of the reference's re-push
                             from every reached vertex: same results, far
                             fewer edges read and counted; 0 (default): the
                             reference's re-push                            */
  uint32_t serve_restarts; /* served loop (sgs_serve): how many times an
                             update may preempt one BFS/SSSP/CC query in
                             flight.  A preempting update is applied at the
                             next round boundary and the queries in flight
                             restart from their sources on the new snapshot
                             (their results and versions are then that
                             snapshot's); once a query in flight has used
                             its restarts, the next update waits for the
                             flight to drain.  0: updates always wait, so
                             every BFS/SSSP/CC query sees exactly the updates
                             that arrived before it.  Default 2            */
} sgs_config;

typedef struct sgs_query_stats {
  uint64_t edges_traversed;   /* edges visited by the last snapshot/start  */
  uint64_t edges_total;       /* since the query was added                 */
  uint64_t invalidated;       /* vertices reset by the last deletion phase */
  uint32_t rounds;            /* relaxation rounds of the last update      */
  uint32_t converged;         /* 1 if the last update converged            */
  double ms;                  /* device time of the last update            */
  double pr_residual_l1;      /* PR: residual L1 when stopped              */
} sgs_query_stats;

typedef struct sgs_engine_stats {
  uint64_t nv;
  uint64_t ne;                /* live edges                                */
  uint64_t slots;             /* used slots (live + tombstones)            */
  uint64_t arena_bytes_hbm;
  uint64_t arena_bytes_host;
  uint64_t hbm_resident_vertices; /* vertices whose block is in HBM        */
  uint64_t last_inserted;     /* kept inserts of the last batch            */
  uint64_t last_deleted;      /* slots tombstoned by the last batch        */
  uint64_t last_relocated;    /* blocks relocated by the last batch        */
  uint64_t repacks;           /* arena repacks so far                      */
  double last_apply_ms;       /* device time of the last graph update      */
  double last_batch_ms;       /* device time of the whole last snapshot    */
  uint64_t kernel_launches;   /* the engine's own kernel launches so far
                                 (CUB sorts and scans not counted)         */
  uint64_t last_batch_edges;  /* edges traversed by all queries in the last
                                 snapshot (sum of their edges_traversed)   */
  /* device edge cache (zero when off) */
  uint64_t cache_lines;       /* capacity in lines of 128 slots            */
  uint64_t cache_resident;    /* lines held after the last admission       */
  uint64_t cache_admissions;  /* admissions so far (one per snapshot, plus
                                 sgs_cache_refresh calls)                  */
  uint64_t last_admitted;     /* lines copied in by the last admission     */
  uint64_t last_evicted;      /* lines evicted by the last admission       */
  uint64_t cache_hit_slots;   /* host-tier slots that BFS/SSSP/CC passes read
                                 from the cache (since load)               */
  uint64_t cache_miss_slots;  /* host-tier slots they read over the host link
                                 (since load)                              */
  uint64_t in_store_bytes;    /* HBM of the in-edge store (0: not built)   */
  uint64_t in_store_builds;   /* transpositions (first use, and rebuilds when
                                 a snapshot's relocations did not fit)     */
  uint64_t bfs_bottom_up_rounds; /* bottom-up BFS rounds run so far        */
  uint64_t host_stagings;     /* explicit copies of the host tier so far   */
  uint64_t last_stage_bytes;  /* bytes of the last one                     */
  uint64_t pr_warm_starts;    /* PageRank starts continued from a previous
                                 query's vector                            */
  uint64_t reclaimed_slots;   /* tombstoned slots reclaimed so far: every
                                 block a snapshot's deletes touch is
                                 compacted in place once its dead slots
                                 reach a sixteenth of its live ones        */
} sgs_engine_stats;

/* Per-kernel-class timing of the relaxation launches (CUDA events on the
 * engine's stream around every launch that has work; off by default).
 * bytes_alg = algorithmic bytes: per walked slot the 4-B id (+4-B weight when
 * a lane needs stored weights) read once for all lanes of a group, per
 * (query, edge) relaxation 8 B of state read+write (PageRank: 16 B FP64
 * residual), plus 20 B per active vertex. */
#define SGS_K_GROUP 0        /* BFS/SSSP/CC relaxation of a query group
                                (its rounds after SGS_K_GROUP_SWEEP's)    */
#define SGS_K_GROUP_INVAL 1  /* parent-tree invalidation of a query group */
#define SGS_K_PR_PUSH 2      /* PageRank residual push                    */
#define SGS_K_WIDE 3         /* relaxation of a wide query group          */
#define SGS_K_WIDE_INVAL 4   /* parent-tree invalidation of a wide group  */
#define SGS_K_PR_PULL 5      /* PageRank sweep as a pull over in-edges    */
#define SGS_K_GROUP_SWEEP 6  /* the first round of a narrow group's phase
                                launched alone on the full grid: after a
                                snapshot's deletions, the re-push from every
                                reached vertex (persistent bit 2)         */
#define SGS_K_COUNT 7
typedef struct sgs_kernel_stats {
  uint64_t launches;
  uint64_t slots;      /* positions walked (edges incl. tombstones)          */
  uint64_t entries;    /* active vertices                                    */
  double bytes_alg;
  double ms;
  uint64_t max_slots;  /* the largest launch (e.g. the all-vertices sweep)   */
  uint64_t max_entries;
  double max_bytes_alg;
  double max_ms;
  uint64_t host_slots;     /* slots of blocks in the pinned-host tier (read
                              over the host link); narrow groups only       */
  uint64_t max_host_slots; /* the same for the largest launch               */
} sgs_kernel_stats;

SGS_API const char *sgs_version(void);
SGS_API const char *sgs_last_error(void);
SGS_API void sgs_config_default(sgs_config *cfg);

SGS_API int sgs_create(const sgs_config *cfg, sgs_engine **out);
SGS_API int sgs_destroy(sgs_engine *e);

/* Graph load.  row has nv+1 entries, col/w row[nv]; w may be NULL unless
 * weight_mode is SGS_W_EXPLICIT.  Lists are taken in the given order. */
SGS_API int sgs_load_csr(sgs_engine *e, uint32_t nv, const uint64_t *row,
                         const uint32_t *col, const uint32_t *w, int mem);
/* Edge list in file order (market_big: parser.cpp:296-406); nv = 0 means
 * max id + 1.  Duplicates and self-loops are kept, like the reference. */
SGS_API int sgs_load_edge_list(sgs_engine *e, uint32_t nv, uint64_t ne,
                               const uint32_t *src, const uint32_t *dst,
                               const uint32_t *w, int mem);
/* Synthetic directed R-MAT generated on the device (2^scale vertices,
 * edge_factor*2^scale draws, self-loops and duplicates removed), weights
 * uniform in [1,64] from wseed in SGS_W_EXPLICIT mode.  Bit-identical to the
 * CPU generator used by the tests. */
SGS_API int sgs_load_rmat(sgs_engine *e, uint32_t scale, uint32_t edge_factor,
                          uint64_t seed, double a, double b, double c,
                          uint64_t wseed);

/* Registers a query and runs it to convergence on the current graph
 * (InitGraph + Start).  source is clamped to [0, nv-1] as the samples do. */
SGS_API int sgs_query_add(sgs_engine *e, int algo, uint32_t source, int *qid);
/* Batched form (no reference counterpart; the reference runs one source per
 * engine): registers n queries at once; the BFS/SSSP/CC ones fill group lanes
 * and each group that received lanes converges all of them in one pass, so
 * many sources share every edge read.  qids[i] receives the i-th id. */
SGS_API int sgs_query_add_many(sgs_engine *e, uint32_t n, const int *algos,
                               const uint32_t *sources, int *qids);
SGS_API int sgs_query_remove(sgs_engine *e, int qid);

/* One snapshot: applies the batch to the graph and brings every registered
 * query up to date incrementally.  Inserts are applied first, then every
 * (src,dst) listed in the deletes is removed (all copies), matching
 * framework.cuh:1011-1012.  ins_w is read only in SGS_W_EXPLICIT mode. */
SGS_API int sgs_apply_batch(sgs_engine *e, const uint32_t *ins_src,
                            const uint32_t *ins_dst, const uint32_t *ins_w,
                            uint64_t n_ins, const uint32_t *del_src,
                            const uint32_t *del_dst, uint64_t n_del, int mem);

/* Re-runs the edge-cache admission now from the current hotness window
 * (without advancing it) and waits until the admitted lines are visible; a
 * no-op when the cache is off.  For drivers that warm the cache after the
 * static run, as the reference's do with LoadCache. */
SGS_API int sgs_cache_refresh(sgs_engine *e);

/* Pipelined snapshots.  sgs_stage_batch copies a batch (pinned host or
 * device arrays) into one of two engine-owned device slots on a copy stream
 * and returns at once; sgs_apply_staged applies the oldest staged batch
 * exactly like sgs_apply_batch.  Staging batch k+1 before applying batch k
 * overlaps its host-to-device copy with snapshot k's work.  The caller keeps
 * the arrays unchanged until the batch has been applied.  At most two
 * batches are staged at a time (SGS_ERR_STATE otherwise). */
SGS_API int sgs_stage_batch(sgs_engine *e, const uint32_t *ins_src,
                            const uint32_t *ins_dst, const uint32_t *ins_w,
                            uint64_t n_ins, const uint32_t *del_src,
                            const uint32_t *del_dst, uint64_t n_del, int mem);
SGS_API int sgs_apply_staged(sgs_engine *e);

/* Copies nv elements of a field (u32, or f64 for PR value/buffer). */
SGS_API int sgs_gather(sgs_engine *e, int qid, int field, void *out, int mem);
SGS_API int sgs_get_query_stats(sgs_engine *e, int qid, sgs_query_stats *out);
SGS_API int sgs_get_engine_stats(sgs_engine *e, sgs_engine_stats *out);

/* Live graph as a CSR (row: nv+1, col/w: ne).  Per-vertex order is not
 * guaranteed.  w may be NULL. */
SGS_API int sgs_graph_export(sgs_engine *e, uint64_t *row, uint32_t *col,
                             uint32_t *w, int mem);
SGS_API int sgs_synchronize(sgs_engine *e);

/* Per-query summary computed on the device (a few bytes to read back per
 * snapshot): out[0] = reached vertices (value != INF; PR: all), out[1] = sum
 * of finite values (PR: sum of ranks as IEEE-754 bits of a double), out[2] =
 * max finite value, out[3] = sum of parents of reached vertices. */
SGS_API int sgs_query_summary(sgs_engine *e, int qid, uint64_t out[4]);
/* The same for n queries with one device-to-host read (out: 4 * n values in
 * query order); the lanes of one narrow group are summarised in one pass. */
SGS_API int sgs_query_summaries(sgs_engine *e, uint32_t n, const int *qids, uint64_t *out);

/* Synthetic update stream (host arrays, no engine needed): n_del distinct
 * existing edges sampled uniformly by edge index and n_ins distinct non-edges
 * (u != v) sampled uniformly over vertex pairs, both w.r.t. the given CSR
 * whose rows must be sorted (e.g. a freshly generated R-MAT graph).  The
 * sequence for (seed, n_ins, n_del) is deterministic; snapshot k takes the
 * k-th slice.  Returns SGS_ERR_INVALID if the graph cannot supply them. */
SGS_API int sgs_gen_update_stream(uint32_t nv, const uint64_t *row,
                                  const uint32_t *col, uint64_t seed,
                                  uint64_t n_ins, uint64_t n_del,
                                  uint32_t *ins_src, uint32_t *ins_dst,
                                  uint32_t *del_src, uint32_t *del_dst);
/* Seeded weights uniform in [1,64] for edge lists (same function as the
 * R-MAT loader's weights). */
SGS_API void sgs_hash_weights(uint64_t wseed, uint64_t n, const uint32_t *src,
                              const uint32_t *dst, uint32_t *w);

/* Readers for the reference's input files (host only; arrays are malloc'd,
 * release them with sgs_free):
 *   edge list "src dst [w]" per line (market_big, parser.cpp:296-406): nv is
 *     max id + 1, edges keep file order; *w is NULL without a third column;
 *   stream sizes "adds dels" per snapshot (Loader.h:27-62);
 *   update file "a|d src dst [w]" lines (Loader.h:64-100); missing weights
 *     read as 0.
 * Blank lines and lines starting with '#' or '%' are skipped. */
SGS_API int sgs_read_edge_list(const char *path, uint32_t *nv, uint64_t *ne,
                               uint32_t **src, uint32_t **dst, uint32_t **w);
SGS_API int sgs_read_stream_sizes(const char *path, uint32_t *nsnap,
                                  uint64_t **adds, uint64_t **dels);
SGS_API int sgs_read_update_file(const char *path, uint64_t *n_add,
                                 uint32_t **add_u, uint32_t **add_v,
                                 uint32_t **add_w, uint64_t *n_del,
                                 uint32_t **del_u, uint32_t **del_v,
                                 uint32_t **del_w);
SGS_API void sgs_free(void *p);

SGS_API int sgs_kernel_timing(sgs_engine *e, int enable);

/* Autotuner (no counterpart in the reference): on the loaded graph, times a
 * probe -- the static convergence of SSSP, BFS and CC from vertex 0 sharing
 * one group -- for each CTAs-per-SM count of the load-balanced relaxation
 * map (4, 8, 16, 32; default 32) and each launch mode (batched rounds or one persistent
 * launch), and keeps the fastest pair for the engine's later work.  The
 * choices change speed only, never results.  Costs 16 static convergences. */
typedef struct sgs_tune {
  uint32_t ctas_per_sm;   /* chosen CTAs per SM of the relaxation map       */
  uint32_t persistent;    /* resulting sgs_config.persistent (bit 0 tuned)  */
  double best_ms;         /* device time of the probe with that choice      */
  uint32_t tried;         /* combinations timed                             */
} sgs_tune;
SGS_API int sgs_autotune(sgs_engine *e, sgs_tune *out);

/* From-scratch SSSP (w != NULL) or BFS (w == NULL) over a CSR that the caller
 * already holds in device memory (row: nv+1 u64 offsets, col/w: row[nv] u32),
 * writing dist[nv] and, if parent != NULL, parent[nv] (device pointers) on
 * `stream` (a cudaStream_t; NULL = default stream).  No counterpart in the
 * reference.  It allocates nothing: for callers that cannot call cudaMalloc
 * (code inside an allocator hook or a memory-pool callback, where an
 * allocation would re-enter the allocator; embedders whose device memory is
 * fixed at start-up), its scratch is a fixed static device array (about
 * 36 MB, reserved on every GPU that loads the library until exit), so nv <=
 * SGS_NOALLOC_MAX_VERTICES and row[nv] <= SGS_NOALLOC_MAX_EDGES, else
 * SGS_ERR_INVALID.  Results equal those of an SGS_SSSP / SGS_BFS query on the
 * same graph (values and smallest-id tight parents).  All calls on a device
 * share the scratch: calls that overlap on the GPU race and must be
 * serialised.  The first call on a device looks up the scratch address; make
 * it before any stream capture starts.  The address is kept for the life of
 * the process, so do not call this on a device after cudaDeviceReset. */
#define SGS_NOALLOC_MAX_VERTICES (1u << 20)
#define SGS_NOALLOC_MAX_EDGES (1ull << 25)
SGS_API int sgs_sssp_csr_noalloc(uint32_t nv, const uint64_t *row,
                                 const uint32_t *col, const uint32_t *w,
                                 uint32_t source, uint32_t *dist,
                                 uint32_t *parent, void *stream);
SGS_API int sgs_get_kernel_stats(sgs_engine *e, int kind, sgs_kernel_stats *out);

/* ---- User algorithms (AppBase functors) on the engine's snapshot path.
 *
 * The reference lets a user write an algorithm as an AppBase<TValue,
 * TBuffer, TWeight> functor struct (include/framework/variants/api.cuh:
 * 22-160) and instantiate Engine<..., TAppImpl, ...> with it
 * (include/framework/framework.cuh:77-140, :389-439).  Here the functor
 * kernels are templates in include/sgs_app.cuh, compiled in the user's own
 * translation unit; the engine (compiled once, in the library) reaches them
 * through these plain-C hooks, so one sgs_apply_batch updates the graph, the
 * built-in queries and every attached user algorithm together.
 *
 * sgs_graph_view: raw device pointers of the current graph layout (valid
 * until the next call that changes the graph: a snapshot, a load).  Block of
 * vertex v: off[v] (bit 63 = pinned-host arena), slots[v] used slots (live
 * edges and tombstones 0xFFFFFFFF), live[v] live out-degree; ids in
 * adj_d/adj_h, weights in wgt_d/wgt_h (explicit mode); cmap/adj_c/wgt_c/cbase
 * describe the device edge cache of the host tier (NULL without one). */
typedef struct sgs_graph_view {
  uint32_t nv;
  int weight_mode;          /* SGS_W_*                                       */
  uint64_t ne;              /* live edges                                    */
  uint64_t slots_total;     /* used slots, tombstones included               */
  uint64_t *off;
  uint32_t *slots, *live, *cap;
  uint32_t *adj_d, *wgt_d, *adj_h, *wgt_h;
  const uint32_t *cmap;
  uint32_t *adj_c, *wgt_c;
  uint64_t cbase;
  void *stream;             /* the engine's cudaStream_t: hooks queue their
                               work on it                                    */
  int device;
  int reserved;
} sgs_graph_view;
SGS_API int sgs_get_graph_view(sgs_engine *e, sgs_graph_view *out);

/* The snapshot as the hooks see it (device arrays, already validated):
 * deletes sorted by (src << 32 | dst); the inserts the engine keeps (sorted,
 * distinct, not deleted in the same snapshot) with their weights (explicit
 * mode; else NULL); their count on the device (*n_ins, at most n_ins_max). */
typedef struct sgs_update_view {
  const uint64_t *del_keys;
  uint64_t n_del;
  const uint64_t *ins_keys;
  const uint32_t *ins_w;
  const uint32_t *n_ins;
  uint64_t n_ins_max;
} sgs_update_view;

/* before_update runs on the old graph, after the batch was validated and
 * before any block changes (the deletion phase: parent-tree invalidation,
 * PageRank-style cancellation); after_update runs on the new graph (the
 * repair and convergence).  Both queue work on g->stream and may
 * synchronise it; a non-zero return fails the snapshot with that status
 * (the graph update itself has happened once before_update returned). */
typedef int (*sgs_app_phase_fn)(void *ctx, const sgs_graph_view *g, const sgs_update_view *u);
typedef struct sgs_app_hooks {
  void *ctx;
  sgs_app_phase_fn before_update;
  sgs_app_phase_fn after_update;
} sgs_app_hooks;
/* Attaches a user algorithm; *app_id identifies it for sgs_app_detach.  The
 * hooks stay attached until detached or the graph is reloaded. */
SGS_API int sgs_app_attach(sgs_engine *e, const sgs_app_hooks *h, int *app_id);
SGS_API int sgs_app_detach(sgs_engine *e, int app_id);
/* Message for sgs_last_error() from a hook that fails. */
SGS_API void sgs_set_last_error(const char *msg);

/* Served request loop (no counterpart in the reference, whose drivers run
 * one source through a fixed snapshot list).  A trace of requests, each with
 * an arrival time in seconds, is served in arrival order on the calling
 * thread, with continuous batching at the granularity of relaxation rounds:
 * BFS/SSSP/CC queries join free lanes of one group kept in flight (at most
 * `slots` lanes in use; 0 = the group's width) between two rounds, so a query
 * arriving while others run starts at the next round boundary and shares
 * their edge passes; a query leaves as soon as no frontier entry carries its
 * lane (summary, and the value / parent vectors when buffers are given, read
 * back) and frees the lane.  An update batch is one snapshot, applied when
 * the flight is empty, so every BFS/SSSP/CC query sees exactly the updates
 * that arrived before it (its `version`).  PageRank queries (no lanes, no
 * source) share one computation per run of consecutive PR requests; updates
 * do not wait for it: a snapshot amends its residual and it continues on the
 * new graph, so a PageRank result reflects at least the updates that arrived
 * before its requests, and its `version` says how many.  With `realtime` the
 * loop waits for arrival times on the wall clock (latency = done_s -
 * arrival_s, queueing included); otherwise every request is taken at once, in
 * arrival order (a closed loop: latency = done_s).  out[i] describes req[i];
 * times are host wall-clock seconds from the start of the call.  Requests
 * that fail carry their status; the call itself fails only for malformed
 * arguments. */
#define SGS_REQ_QUERY 0
#define SGS_REQ_UPDATE 1
typedef struct sgs_request {
  int kind;                 /* SGS_REQ_QUERY or SGS_REQ_UPDATE               */
  int algo;                 /* query: SGS_BFS / SGS_SSSP / SGS_CC / SGS_PR   */
  uint32_t source;          /* query source                                  */
  uint32_t reserved;
  double arrival_s;         /* >= 0                                          */
  void *value_out;          /* query, optional host buffer: nv u32, PR: nv
                               double                                        */
  uint32_t *parent_out;     /* query, optional host buffer: nv u32           */
  const uint32_t *ins_src, *ins_dst, *ins_w;  /* update: host arrays        */
  const uint32_t *del_src, *del_dst;
  uint64_t n_ins, n_del;
} sgs_request;
typedef struct sgs_completion {
  int status;               /* SGS_OK or this request's error                */
  uint32_t batch;           /* queries: lanes in flight when it joined (PR:
                               requests sharing the computation); 1 for an
                               update                                        */
  uint64_t version;         /* query: the snapshot its result reflects (the
                               updates applied before its last run; PR: at
                               least those before it arrived); an update:
                               its own position in the sequence             */
  double start_s, done_s;   /* seconds from the start of the call            */
  uint64_t summary[4];      /* query: as sgs_query_summary                   */
  uint64_t edges;           /* edges traversed for this request (a restarted
                               query: its last run only)                     */
  uint32_t restarts;        /* query: times an update restarted it           */
  uint32_t reserved;
} sgs_completion;
SGS_API int sgs_serve(sgs_engine *e, const sgs_request *req, uint32_t n,
                      uint32_t slots, int realtime, sgs_completion *out);

/* Differentiable weighted personalized PageRank (FP64).  Generalises the
 * reference's PageRank fixed point (samples/hybrid_pr/hybrid_pr.cu:26-151,
 * x = (1-alpha) + alpha * sum_{u->v} x_u / outdeg_u, dangling mass dropped)
 * to edge weights w (P[u,v] = w_uv / sum_v' w_uv') and K teleport vectors:
 *     X[:,k] = (1-alpha) T[:,k] + alpha P^T X[:,k]
 * With T = 1 and unit weights X is the reference's PageRank.  The backward
 * pass has no counterpart in the reference.  Layout: X, T, G, gT are
 * vertex-major [nv][K] doubles; w and gw are per edge in the CSR order of
 * the prepared graph (sgs_ppr_export).  `mem` says where all arrays live.
 * Convergence: Jacobi steps until the L1 change summed over all nv*K entries
 * is below tol; SGS_ERR_NOCONV after max_iter steps.  *iters (optional) gets
 * the steps taken.  Weights must be positive and finite (else
 * SGS_ERR_INVALID).  A handle is not thread-safe. */
typedef struct sgs_ppr sgs_ppr;
SGS_API int sgs_ppr_create_csr(int device, uint32_t nv, const uint64_t *row,
                               const uint32_t *col, int mem, sgs_ppr **out);
/* Prepares the engine's current graph (a snapshot of the dynamic graph). */
SGS_API int sgs_ppr_create(sgs_engine *e, sgs_ppr **out);
SGS_API int sgs_ppr_destroy(sgs_ppr *p);
SGS_API int sgs_ppr_info(sgs_ppr *p, uint32_t *nv, uint64_t *ne);
SGS_API int sgs_ppr_export(sgs_ppr *p, uint64_t *row, uint32_t *col, int mem);
SGS_API int sgs_ppr_forward(sgs_ppr *p, const double *w, const double *T,
                            uint32_t K, double alpha, double tol,
                            uint32_t max_iter, double *X, int *iters, int mem);
/* Adjoint for the upstream gradient G = dL/dX of a forward result X:
 *     Y = G + alpha P Y,  gT = dL/dT = (1-alpha) Y,
 *     gw[e=(u,v)] = dL/dw_uv = sum_k X[u,k] (alpha Y[v,k] - Y[u,k] + G[u,k]) / s_u
 * gw or gT may be NULL to skip them. */
SGS_API int sgs_ppr_backward(sgs_ppr *p, const double *w, const double *X,
                             const double *G, uint32_t K, double alpha,
                             double tol, uint32_t max_iter, double *gw,
                             double *gT, int *iters, int mem);
/* Device timing of the last forward/backward call (CUDA events on the
 * handle's stream).  steps_ms is filled only while sgs_ppr_timing is on
 * (events around every Jacobi step).  bytes_alg_step = algorithmic bytes of
 * one step: per edge the 4-B neighbour id, 8-B probability and 8K-B neighbour
 * row; per vertex 16 B of offsets and 24K B of state (B, x read; out written). */
typedef struct sgs_ppr_stats {
  int32_t iters;             /* Jacobi steps of the last call              */
  uint32_t pieces_in;        /* work pieces of hub vertices, CSC and CSR   */
  uint32_t pieces_out;
  uint32_t reserved;
  double ms;                 /* device time of the whole last call         */
  double steps_ms;           /* device time of its Jacobi steps            */
  double bytes_alg_step;
  uint64_t kernel_launches;  /* own kernel launches since the handle was made */
} sgs_ppr_stats;
SGS_API int sgs_ppr_timing(sgs_ppr *p, int enable);
SGS_API int sgs_ppr_get_stats(sgs_ppr *p, sgs_ppr_stats *out);

#ifdef __cplusplus
}
#endif
#endif /* SGS_H */
