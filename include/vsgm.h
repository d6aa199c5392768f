/* vsgm_b200 C ABI: B200-native subgraph enumeration/counting.
 *
 * The reference (VSGM) has no FFI layer; its operator surface is the
 * pm_pipeline command line plus the in-process PipelineExecutor class.  Every
 * entry point below names the reference interface it replaces (file:line within
 * the reference project).  All functions return 0 on success and a negative code
 * on failure; vsgm_last_error / vsgm_engine_error give the message.  Nothing here
 * exits the process.  Plain pointers and sizes only; the caller owns every
 * buffer it passes in.
 */
#ifndef VSGM_H
#define VSGM_H

#include <stddef.h>
#include <stdint.h>

#include "vsgm_plan.h"

#ifdef __cplusplus
extern "C" {
#endif

#define VSGM_OK 0
#define VSGM_EINVAL (-1)   /* bad argument */
#define VSGM_EIO (-2)      /* file error */
#define VSGM_ECUDA (-3)    /* CUDA runtime error */
#define VSGM_ENOMEM (-4)   /* HBM budget or host memory exhausted */
#define VSGM_ETIMEOUT (-5) /* a bounded device wait gave up */

/* Message of the last failed host-side call on this thread. */
const char* vsgm_last_error(void);

/* ------------------------------------------------------------------ planning */

/* Pattern((PresetPatternType)id, false) + Plan::Optimize
 * (src/query/pattern.h:31-380, src/query/plan.h:548-561; pm_pipeline -p,
 * src/app/pattern_matching_pipeline.cu:69,79-80).  id in 0..18. */
int vsgm_plan_pattern(int pattern_id, vsgm_plan* out);

/* Clique(k) + Plan::Optimize (src/query/clique.h:9-37; pm_pipeline -kc,
 * src/app/pattern_matching_pipeline.cu:61).  k in 3..7. */
int vsgm_plan_clique(int k, vsgm_plan* out);

/* Query(n, e, adj) + Plan::Optimize (src/query/query.h:62-78): adj_bits[i] bit j
 * set iff pattern edge (i, j); the pattern must be connected, n in 2..7. */
int vsgm_plan_query(int n, const uint8_t* adj_bits, vsgm_plan* out);

/* Graphlet(k)->GetQueries() + Plan::Optimize per query (src/query/graphlet.h:15-136;
 * pm_pipeline -km, src/app/pattern_matching_pipeline.cu:64-66).  Writes at most cap
 * plans and the total number of graphlets to *n_out. */
int vsgm_plan_graphlets(int k, vsgm_plan* out, int cap, int* n_out);

/* The plan of the same query with the search sequence taken from seq[0..n-1]
 * instead of Plan::GenerateSearchSequence (src/query/plan.h:210-265); every later
 * table is derived as Plan::Optimize derives it.  The learned planner's hook. */
int vsgm_plan_reorder(const vsgm_plan* base, const uint8_t* seq, vsgm_plan* out);

/* |Aut(P)| of a planned pattern. */
uint64_t vsgm_plan_automorphisms(const vsgm_plan* p);

/* ------------------------------------------------------------ graphs and files */

/* Release memory this library allocated for the caller. */
void vsgm_free(void* p);

/* GraphIO::ReadCSRBinFile (src/graph/graph_io.h:57-100), as parallel bulk reads
 * (the reference reads one element per fread).  The file size must match its
 * header exactly.  *row_ptrs (V+1 entries) and *cols (E entries) are allocated
 * here: vsgm_free. */
int vsgm_read_csr_bin(const char* path, uint64_t* V, uint64_t* E, uint64_t** row_ptrs, uint32_t** cols);

/* The same reader in two steps, for callers that own the buffers (pinned host
 * memory, for instance): the header (sizes checked against the file), then the
 * arrays straight into row_ptrs[V+1] and cols[E] with `threads` parallel reads
 * (0 = all cores). */
int vsgm_csr_bin_header(const char* path, uint64_t* V, uint64_t* E);
int vsgm_read_csr_bin_into(const char* path, uint64_t V, uint64_t E, uint64_t* row_ptrs, uint32_t* cols, int threads);

/* GraphIO::WriteCSRBinFile (src/graph/graph_io.h:313-339). */
int vsgm_write_csr_bin(const char* path, uint64_t V, uint64_t E, const uint64_t* row_ptrs, const uint32_t* cols);

/* ViewBinManager::LoadViewBinPartition's file read (src/view/view_bin_manager.h:30-41). */
int vsgm_read_vbmap(const char* path, uint64_t V, int32_t* bins, int32_t* n_bins);
int vsgm_write_vbmap(const char* path, uint64_t V, const int32_t* bins, int32_t n_bins);

/* GraphIO::Validate (src/graph/graph_io.h:416-444) minus the dangling-vertex
 * rule: number of self loops, out-of-range, unsorted or duplicate entries. */
uint64_t vsgm_csr_defects(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols);

/* Synthetic inputs (the reference reads SNAP/Friendster files instead).  Output
 * arrays are allocated here: vsgm_free.  threads <= 0 uses every host core. */
int vsgm_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int threads, uint64_t* V, uint64_t* E,
                  uint64_t** row_ptrs, uint32_t** cols);
int vsgm_gen_chung_lu(uint64_t V, uint64_t target_edges, double gamma, uint64_t max_degree, uint64_t seed, int threads, uint64_t* E,
                      uint64_t** row_ptrs, uint32_t** cols);
/* connected random pattern (n in [n_min, n_max], edge probability p) from stream
 * seed at *counter; advances *counter. */
int vsgm_random_pattern(int n_min, int n_max, double p, uint64_t seed, uint64_t* counter, int* n, uint8_t* adj_bits);

/* Degree-ordered relabelling of a whole graph (no reference counterpart; the
 * reference keeps the input's ids).  new id = rank of (degree, old id), ascending
 * when `ascending`, else descending; new_of_old[V], row_ptrs_out[V+1], cols_out[E]
 * are caller-allocated.  Exact total counts are invariant to relabelling; apply
 * the same permutation to a .vbmap (bins_new[new_of_old[v]] = bins[v]). */
int vsgm_degree_relabel(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, int ascending, int threads, uint32_t* new_of_old,
                        uint64_t* row_ptrs_out, uint32_t* cols_out);

/* ViewBin::Materialize (src/view/view_bin.h:66-142): full-V CSR holding the
 * adjacency rows of every source with degree >= root_degree (all when 0) and of
 * every vertex within hop-1 steps of one.  view_row_ptrs has V+1 entries; fails
 * with VSGM_ENOMEM (and *n_cols set) if more than cols_cap entries are needed. */
int vsgm_view_materialize(uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, const uint32_t* sources, uint64_t n_sources, int hop,
                          uint64_t root_degree, int threads, uint64_t* view_row_ptrs, uint32_t* view_cols, uint64_t cols_cap, uint64_t* n_cols);

/* ------------------------------------------- view-bin tools on the device
 * The offline chain that produces the .vbmap (features -h 1 -> kmeans ->
 * view_packing), run on GPU `device` from host buffers, each with exactly the
 * reference tool's output.  The graph must be undirected with sorted rows. */

/* features -h 1 (src/tools/features.cc:177-201): every row gains its own vertex
 * in sorted position.  out_row_ptrs has V+1 entries, out_cols E+V. */
int vsgm_features_1hop(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t* out_row_ptrs, uint32_t* out_cols);

/* kmeans -k K -i max_iter -init 1 [-rc 1] (src/tools/kmeans.cc:54-247, 386-510,
 * 636-694; cosine similarity, src/tools/kmeans_utils.h:40-160), single level.
 * The random initialisation is given explicitly: starts[p] (n_starts = the
 * reference's thread count -t) is the cluster its thread p draws with
 * std::rand() % K (kmeans.cc:125-141); thread p's vertices p, p+T, ... take
 * consecutive clusters from there.  With -rc 1 the clusters are renumbered by
 * the non-zero entries of their centroids, counted for the first
 * min(K, n_starts) only, as the reference counts them.  Writes the
 * assignment (V entries, empty clusters removed), the sizes of the n_clusters
 * non-empty clusters (K entries of space) and *n_clusters.  K <= 128. */
int vsgm_kmeans(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, int K, int max_iter, const int32_t* starts, int n_starts,
                int reorder_centroids, int32_t* assignment, int64_t* cluster_sizes, int32_t* n_clusters);

/* view_packing -s 1 (src/tools/view_packing.cc:141-324, ViewBinPool with one
 * open bin, src/tools/view_bin.h:22-138): each of the n_seqs sequences
 * order[seq_offsets[q] .. seq_offsets[q+1]) (one per packing thread -t; their
 * order built from the partition file as the reference builds it) is packed
 * next-fit into bins of at most max_bin_size row entries, a source adding the
 * rows of its (hop-1)-ball not yet in the bin (hop 1..3); then the bins are
 * merged next-fit by size.  Writes the .vbmap content (bin_of_vertex[V],
 * *n_bins) and, when bin_sizes is given, the row entries of the first
 * sizes_cap merged bins (the .vbstat sizes).  A source whose ball alone
 * exceeds max_bin_size is an error (the reference drops it and fails its own
 * vertex-count assertion). */
int vsgm_view_packing(int device, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, const uint32_t* order, const uint64_t* seq_offsets,
                      int n_seqs, int hop, uint64_t max_bin_size, int32_t* bin_of_vertex, int32_t* n_bins, uint64_t* bin_sizes, uint64_t sizes_cap);

/* ------------------------------------------------------------------- engine */

typedef struct vsgm_engine vsgm_engine; /* one per host thread per GPU */

/* PipelineExecutor(device_id, graph, plans, max_partitioned_sources_num)
 * (src/executor/pipeline_executor.h:22-47).  hbm_budget_bytes bounds the
 * engine's working memory (0 = 90% of free HBM; the reference hard-codes
 * 10.6 GiB at src/common/meta.h:29-36). */
int vsgm_create(int device, uint64_t V, const vsgm_plan* plans, int n_plans, uint64_t max_sources, uint64_t hbm_budget_bytes, vsgm_engine** out);

/* PipelineExecutor::Transfer (src/executor/pipeline_executor.h:64-81): copy one
 * view (full-V CSR + its sources) from host memory to the device.  The host
 * buffers may be reused as soon as the call returns. */
int vsgm_transfer_view(vsgm_engine* e, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols, const uint32_t* sources, uint64_t n_sources);

/* PipelineExecutor::Transfer overlapped with matching (the reference copies
 * synchronously, src/executor/pipeline_executor.h:64-81).  The view travels in
 * compact form: the ascending ids of its vertices with a non-empty row
 * (vertices[n_vertices]) and their offsets into cols (offsets[n_vertices+1],
 * offsets[0] = 0) - 12 bytes per row of the view instead of 8 per vertex of the
 * graph; vsgm_view_compact derives it from a full-V view.  The copies go to the
 * engine's second view buffer on its copy stream and the call returns at once, so
 * they run while the current view is matched; with host buffers from
 * vsgm_host_alloc (pinned) they are truly asynchronous.  The host buffers must stay
 * untouched until vsgm_view_released returns.  vsgm_swap_view makes the prefetched
 * view the current one (the engine's stream waits for the copies; the host does
 * not).  One prefetch at a time. */
int vsgm_prefetch_view(vsgm_engine* e, const uint32_t* vertices, uint64_t n_vertices, const uint64_t* offsets, const uint32_t* cols,
                       const uint32_t* sources, uint64_t n_sources);
int vsgm_view_released(vsgm_engine* e);
int vsgm_swap_view(vsgm_engine* e);
/* compact form of a full-V view (row_ptrs[V+1], rows contiguous from 0): *n_vertices
 * rows listed; vertices and offsets need room for V and V+1 entries */
int vsgm_view_compact(uint64_t V, const uint64_t* row_ptrs, uint32_t* vertices, uint64_t* offsets, uint64_t* n_vertices);
/* pinned host memory (cudaMallocHost) for view buffers, and its release */
int vsgm_host_alloc(uint64_t bytes, void** out);
int vsgm_host_free(void* p);

/* Bind a view already resident in device memory on the engine's device (no
 * copy; the caller keeps it alive until the next transfer or destroy). */
int vsgm_bind_view_device(vsgm_engine* e, const uint64_t* d_row_ptrs, const uint32_t* d_cols, uint64_t n_cols, const uint32_t* d_sources, uint64_t n_sources);

/* Keep the whole graph resident on the engine's device (row_ptrs[V+1], cols)
 * so that views can be built there: replaces the host producers of
 * src/app/pattern_matching_pipeline.cu:117-150 (one LoadViewBin per bin).  With the
 * engine option "relabel" set, the graph (undirected: both directions stored) is
 * relabelled on the device so that ids ascend with (degree, id) - the permutation
 * of vsgm_degree_relabel - and the sources given to vsgm_graph_view /
 * vsgm_materialize_view stay in the caller's ids; totals do not change, and
 * vsgm_read_view then returns the relabelled rows. */
int vsgm_upload_graph(vsgm_engine* e, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols);

/* ViewBin::Materialize (src/view/view_bin.h:66-142) on the device from the
 * uploaded graph: the halo of the sources (degree >= root_degree, all when 0)
 * within hop-1 steps gets its full rows; the result becomes the current view
 * with exactly these sources, byte-identical to vsgm_view_materialize. */
int vsgm_materialize_view(vsgm_engine* e, const uint32_t* sources, uint64_t n_sources, int hop, uint64_t root_degree);

/* The uploaded graph itself becomes the current view, with these sources as
 * roots: every row is present, so no halo is built.  Counts equal those over
 * the sources' k-hop halo (a match rooted at a source reads only rows inside
 * its halo).  No reference counterpart: the reference never holds the whole
 * graph on the GPU. */
int vsgm_graph_view(vsgm_engine* e, const uint32_t* sources, uint64_t n_sources);

/* Copy the current view back to the host (row_ptrs[V+1], cols[cols_cap]);
 * VSGM_ENOMEM with *n_cols set when cols_cap is too small.  No reference
 * counterpart (inspection of a device-built view). */
int vsgm_read_view(vsgm_engine* e, uint64_t* row_ptrs, uint32_t* cols, uint64_t cols_cap, uint64_t* n_cols);

/* PipelineExecutor::Match (src/executor/pipeline_executor.h:83-109): run every
 * plan over every source of the current view and add to the per-plan totals. */
int vsgm_match(vsgm_engine* e);

/* PipelineExecutor::GetTotalCounts (src/executor/pipeline_executor.h:62):
 * n_plans exact uint64 totals accumulated since create / reset. */
int vsgm_get_counts(vsgm_engine* e, uint64_t* out);
int vsgm_reset_counts(vsgm_engine* e);

/* Per-plan execution statistics of the last vsgm_match (no reference
 * counterpart; the reference prints timings only). */
typedef struct vsgm_plan_stats {
  uint64_t op_paths[VSGM_MAX_OPS];    /* partial matches entering each op */
  uint64_t op_outputs[VSGM_MAX_OPS];  /* candidates / children / count produced */
  double op_ms[VSGM_MAX_OPS];         /* device time per op (CUDA events) */
  uint64_t op_launches[VSGM_MAX_OPS]; /* kernels launched per op */
  uint64_t op_bytes[VSGM_MAX_OPS];    /* algorithmic bytes per op */
  uint64_t batches;                   /* memory-bounded batches executed */
  uint64_t peak_bytes;                /* peak working memory */
} vsgm_plan_stats;
int vsgm_get_stats(vsgm_engine* e, int plan, vsgm_plan_stats* out);

/* Batched execution (no reference counterpart: the reference runs one plan at a
 * time over one view, src/executor/pipeline_executor.h:83-109).  vsgm_add_view
 * uploads another view (its own vertex count) and keeps it resident;
 * vsgm_run_batched runs every (plan, view) pair of the given ids in ONE
 * persistent launch fed by a device work queue of root ranges, and writes
 * counts[p * n_views + v] (exact uint64). */
int vsgm_add_view(vsgm_engine* e, uint64_t V, const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n_cols, const uint32_t* sources,
                  uint64_t n_sources, int* view_id);
int vsgm_run_batched(vsgm_engine* e, const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t* counts);

/* The same persistent (hybrid) run over an explicit list of (plan, view) pairs,
 * e.g. a different plan of one pattern per view; counts[i] for pair i. */
int vsgm_run_pairs(vsgm_engine* e, const int* plan_ids, const int* view_ids, int n_pairs, uint64_t* counts);

/* vsgm_run_batched plus, per (plan, view) pair: level_paths[pair * VSGM_MAX_OPS + i]
 * = partial matches entering op i (the intermediate sizes the learned planner is
 * trained on), and with step_budget > 0 every task stops after that many steps and
 * sets overflow[pair] (its counts are then partial).  Either output may be NULL. */
int vsgm_run_batched_ex(vsgm_engine* e, const int* view_ids, int n_views, const int* plan_ids, int n_plans, uint64_t step_budget, uint64_t* counts,
                        uint64_t* level_paths, uint32_t* overflow);

typedef struct vsgm_batch_stats {
  uint64_t tasks;         /* root-range tasks in the last batched run */
  uint64_t launches;      /* kernels launched by it */
  uint64_t scratch_bytes; /* per-warp scratch allocated */
  double ms;              /* device time (with profiling on) */
  uint64_t level_pairs;   /* (plan, view) pairs the hybrid run counted level-wise */
} vsgm_batch_stats;
int vsgm_get_batch_stats(vsgm_engine* e, vsgm_batch_stats* out);

/* ------------------------------------------------------------- learned planner
 * No reference counterpart: the reference's only order heuristic is
 * Plan::GenerateSearchSequence (src/query/plan.h:210-265).  A 3-layer MLP
 * (n_in -> n_hidden -> n_hidden -> n_out, ReLU) whose GEMMs take BF16 operands
 * and accumulate in FP32, trained with Adam on FP32 master weights.  Parameters
 * are packed W1[n_in][n_hidden], b1, W2[n_hidden][n_hidden], b2,
 * W3[n_hidden][n_out], b3.  Host arrays are row-major float. */
typedef struct vsgm_mlp vsgm_mlp;
int vsgm_mlp_create(int device, int n_in, int n_hidden, int n_out, uint64_t seed, vsgm_mlp** out);
uint64_t vsgm_mlp_num_params(vsgm_mlp* m);
int vsgm_mlp_get_params(vsgm_mlp* m, float* host);
int vsgm_mlp_set_params(vsgm_mlp* m, const float* host);
int vsgm_mlp_forward(vsgm_mlp* m, const float* x, int batch, float* y);
/* masked MSE loss and its gradient w.r.t. every parameter (packed like the params) */
int vsgm_mlp_gradients(vsgm_mlp* m, const float* x, const float* target, const float* mask, int batch, float* loss, float* grads);
int vsgm_mlp_train_step(vsgm_mlp* m, const float* x, const float* target, const float* mask, int batch, float lr, float* loss);
const char* vsgm_mlp_error(vsgm_mlp* m);
int vsgm_mlp_destroy(vsgm_mlp* m);

/* Tuning knobs (no reference counterpart), for every plan or for one plan:
 *   "clique_bits" (default 1): a 3- or 4-clique plan (complete pattern, every pair
 *   of vertices ordered, the root first) counts at each root the cliques of its
 *   out-neighbourhood from bit rows of that neighbourhood's adjacency in shared
 *   memory; roots with more than 1024 neighbours above them run the plan;
 *   "edge_triangles" (default 1): the diamond plan (-p 2) is counted from per-edge
 *   triangle counts (each triangle found once, at its smallest vertex) as the sum
 *   over the root's edges to larger neighbours of the pairs of common neighbours;
 *   a view with a vertex of more than 16384 neighbours above it runs the plan;
 *   "relabel" (engine-wide, default 0): vsgm_upload_graph orders the resident
 *   graph's ids by degree on the device (see there);
 *   "fuse_tail" (default 1): a MATERIALIZE followed by the final COMPUTE_COUNT runs as
 *   one kernel that stages the parent's shared lists in shared memory instead of
 *   expanding the children;
 *   "stage_cap" (default and maximum 1536): largest shared list staged per warp, in
 *   vertex ids; larger ones take the per-child intersection;
 *   "merge_ratio" (default 4): two lists whose restricted lengths are within this
 *   ratio are intersected by a coalesced merge, otherwise by galloping (0: always
 *   gallop);
 *   "c4_aggregate" (default 1): a 4-cycle pattern is counted by wedge aggregation
 *   rooted at each cycle's largest vertex (sum over opposite vertices of
 *   C(wedges, 2)) instead of the plan's op sequence; totals are identical, per-view
 *   counts are attributed to the largest instead of the smallest vertex;
 *   "walk_ratio" (default 8): in the fused tail a child with a long slice of the
 *   staged set walks its own adjacency range coalesced (probing the stage) unless
 *   that range is this many times longer than the slice, then it gallops (0: always
 *   gallop);
 *   "lane_slice" (default 16): in the fused tail a child whose slice of the staged
 *   set is at most this long is handled by one lane, longer ones by the whole warp;
 *   "tail_merge" (default 0): in the fused tail a heavy child intersects its slice
 *   and its part of N(c) by a merge-path split over the warp's lanes instead of
 *   the walk / gallop;
 *   "c4_heavy" (default 12289): roots with at least this many wedges are counted by
 *   groups sharing the whole GPU with L2-resident counters (0: every root);
 *   "c4_window" (default 0): heavy roots with fewer than 65536 lower neighbours count
 *   the wedges ending in the 393,216 ids just below them in the distributed shared
 *   memory of a 4-block cluster, the rest in the groups (measured slower on R-MAT 22);
 *   "c4_balance" (default 0): a heavy group's wedge launch splits its centres'
 *   adjacency entries evenly over the warps instead of giving each warp whole
 *   centres (faster per launch alone, slower in the two-stream group pipeline on
 *   R-MAT 22);
 *   "c4_hash" (default 1): the other roots keep their counters in a shared-memory
 *   hash table (a warp per root up to 768 wedges, a block up to 12288; beyond, and
 *   with 0, one block per root with dense counters in HBM);
 *   "set_reuse" (default 1): a COMPUTE directly followed by the final COMPUTE_COUNT
 *   of a vertex with the same backward lists and conditions (the diamond's tail)
 *   counts the pairs of one intersection instead of intersecting twice;
 *   "lane_merge" (default 0): counting kernels merge two such lists with each lane
 *   walking its own chunk instead of 32-element warp windows;
 *   "hybrid_steps" (engine-wide, default 2^14): vsgm_run_batched runs every pair in
 *   the persistent launch with this per-task step bound and counts the pairs it
 *   stopped again with the level-wise engine on their resident view (0: the
 *   persistent launch alone, unbounded);
 *   "streams" (engine-wide, default 4): the pairs a hybrid batched run recounts
 *   level-wise run this many at a time, each on its own stream and host thread with
 *   a slice of the engine's working memory (1: one after the other);
 *   "root_stride" (engine-wide, default 1): match only every k-th source of the view
 *   (the autotuner's samples; counts are then those of the sample);
 *   "only_plan" (engine-wide, default -1): vsgm_match runs only this plan.
 * None of the knobs changes a total count. */
int vsgm_set_plan_option(vsgm_engine* e, int plan, const char* name, int64_t value);
int vsgm_set_option(vsgm_engine* e, const char* name, int64_t value);

/* Collect op_ms / op_bytes (adds CUDA events and a small accounting pass). */
int vsgm_set_profiling(vsgm_engine* e, int on);

/* Engine stream (cudaStream_t) for callers that order their own work with it. */
void* vsgm_engine_stream(vsgm_engine* e);

const char* vsgm_engine_error(vsgm_engine* e);

/* Allocation-free counting.  This entry point has no counterpart in the
 * reference.  It is for callers that may not allocate device memory - code that
 * runs under a pool or allocator owning all of the process's device memory, or that
 * must have a fixed footprint known before it runs: it counts one plan over one
 * view already in device memory (d_row_ptrs[V+1], d_cols, d_sources[n_sources]) and
 * writes the exact count to *count (host memory), using the same persistent kernel
 * as vsgm_run_batched but with all of its working buffers inside one 48 MiB
 * file-scope device array, which every GPU that loads this library holds until the
 * process exits.  It calls no cudaMalloc or cudaFree.  The first call on a device
 * looks up the array's device address (make that first call before any stream
 * capture); the address is kept per device together with the id of the context
 * it belongs to, and looked up again when the device's context has changed (after
 * cudaDeviceReset, the rebuilt context loads the array anew, possibly elsewhere), so
 * the first call after such a reset also belongs before any capture.  Limit: plan ops x the view's maximum degree <= 24,319; larger views
 * are rejected with VSGM_EINVAL and a message.  The array is shared by every call on
 * the device and keeps the last call's contents (each call clears what it needs):
 * calls that overlap on the GPU race, so serialise them.  stream may be NULL (the
 * legacy default stream); the call returns after the stream is synchronised. */
int vsgm_count_noalloc(int device, const vsgm_plan* plan, uint64_t V, const uint64_t* d_row_ptrs, const uint32_t* d_cols, const uint32_t* d_sources,
                       uint64_t n_sources, void* stream, uint64_t* count);

/* ~PipelineExecutor (src/executor/pipeline_executor.h:48-54). */
int vsgm_destroy(vsgm_engine* e);

#ifdef __cplusplus
}
#endif

#endif
