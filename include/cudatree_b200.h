/*
 * cudatree_b200 — C ABI of the B200 random-forest fit + predict engine.
 *
 * Every entry point returns an int status (CT_OK == 0); ct_last_error() gives
 * the text of the last failure on the calling thread.  Pointers named *_dev
 * or documented as device pointers are CUDA device memory owned by the caller;
 * `stream` is a cudaStream_t (NULL = legacy default stream).  The library
 * allocates no device memory on these paths: callers size a workspace with
 * the matching *_workspace_size call and pass it in.  The only objects the
 * library owns across calls are the opaque handles of the serving engine.
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the EasonLiao/CudaTree source tree).
 */
#ifndef CUDATREE_B200_H
#define CUDATREE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CT_OK = 0,
  CT_ERR_ARG = 1,         /* invalid argument or size                      */
  CT_ERR_OOM = 2,         /* workspace too small / device memory exhausted  */
  CT_ERR_CUDA = 3,        /* a CUDA runtime call failed                     */
  CT_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up             */
  CT_ERR_UNSUPPORTED = 5, /* shape outside the supported limits             */
  CT_ERR_INTERNAL = 6,    /* device-side consistency check failed           */
  CT_ERR_CAPACITY = 7     /* tree node capacity exceeded                    */
};

enum { CT_FIT_PLAIN = 0, CT_FIT_BATCHED = 1 };

/* Limits of this build. */
#define CT_MAX_CLASSES 1024u
#define CT_MAX_FEATURES 65536u

/* Training problem.  Device pointers.  Replaces the state fit_init builds
 * (cudatree/random_forest.py:215-266): feature-major samples (:233), compacted
 * labels (:85-99, :220), presorted indices (:247-248), dtype choice (:224-230). */
typedef struct ct_problem {
  const float* x_fm;          /* [n_features][n_rows] float32                    */
  const void* labels;         /* [n_rows] class ids, uint8 or uint16             */
  const void* presort;        /* [n_features][n_rows] stable ascending row order */
  uint32_t n_rows;
  uint32_t n_features;
  uint32_t n_classes;
  uint32_t index_bytes;       /* 2 (n_rows <= 65535) or 4                        */
  uint32_t label_bytes;       /* 1 (n_classes <= 255) or 2                       */
  uint32_t max_features;      /* features examined per node                      */
  uint32_t min_samples_split; /* random_forest.py:47                             */
  uint32_t bootstrap;         /* random_forest.py:48                             */
  uint64_t seed;              /* forest seed for all random streams              */
} ct_problem;

/* Double-buffered per-tree index lists (reference sorted_indices_gpu and
 * sorted_indices_gpu_, random_tree.py:466-467).  Slot s, buffer b, feature f
 * starts at si[b] + ((size_t)s * n_features + f) * stride elements.  mark
 * holds the [n_slots][n_rows] byte mark table (reference mark_table,
 * random_forest.py:168; the bootstrap's in-bag marks) followed, at the next
 * 256-byte boundary, by the packed [n_slots][bit_words] uint32 flags that
 * the partition reads: scratch of each partition call, which clears them
 * and sets the left rows of its splits (a forest queue's batch sets left
 * rows and clears right ones); ct_mark_bytes gives the size. */
/* The partition and compaction kernels copy index tiles with 16-byte TMA
 * bulk copies and may read up to 15 bytes past the last element of the
 * si0/si1 buffers and of the presort: allocate them with >= 16 bytes of
 * readable padding. */
typedef struct ct_lists {
  void* si0;
  void* si1;
  uint8_t* mark;
  uint32_t stride;
  uint32_t n_slots;
} ct_lists;

/* One tree node waiting for a split (reference queue entry idx_array /
 * si_idx_array / nid_array, random_tree.py:617-621). 32 bytes. */
typedef struct ct_node {
  uint32_t slot;     /* tree slot holding the node's lists                 */
  uint32_t start;    /* first position of the node in every feature list   */
  uint32_t n;        /* samples in the node                                */
  uint32_t raw_id;   /* node id in the slot's raw tree arrays              */
  uint64_t key;      /* path key (selects the node's feature subset)       */
  float impurity;    /* impurity reported by the parent split (root 1.0)   */
  uint32_t buf;      /* which index-list buffer holds the node (0 or 1)    */
} ct_node;

/* Best split of one node (reference find_min_imp output, dfs_module.cu:202-206,
 * plus the threshold of random_tree.py:641-644). 32 bytes. */
typedef struct ct_split_result {
  double score;       /* imp_left + imp_right in fp64; +inf if none        */
  uint32_t feature;   /* chosen feature, 0xffffffff if none                */
  uint32_t pos;       /* last position of the left child in that feature   */
  float imp_left;
  float imp_right;
  float threshold;
  uint32_t n_selected; /* non-constant features examined                   */
} ct_split_result;

/* Raw tree storage for n_slots trees, nodes in allocation order.  Replaces
 * the per-tree node arrays of random_tree.py:284-289. */
typedef struct ct_tree_buffers {
  uint32_t* left;      /* [n_slots][capacity], 0 = leaf                    */
  uint32_t* right;
  uint32_t* feature;
  float* threshold;
  uint32_t* value;     /* leaf class id                                    */
  uint32_t* n_nodes;   /* [n_slots]                                        */
  uint32_t capacity;   /* >= 2 * n_rows                                    */
} ct_tree_buffers;

typedef struct ct_fit_options {
  uint32_t mode;            /* CT_FIT_PLAIN or CT_FIT_BATCHED                       */
  uint32_t bfs_threshold;   /* plain: nodes with n <= this go to the BFS queue
                               (random_tree.py:616-622); 0 = reference formula     */
  uint32_t subtree_cutoff;  /* nodes with n <= this are grown whole by one warp
                               (<= 128; 0 disables); the trees do not change        */
  uint32_t scan_piece;      /* elements per split-scan work item (0 = default)      */
  uint32_t flags;           /* CT_FIT_PROFILE | CT_FIT_HOST_LOOP                    */
  uint32_t step_nodes;      /* nodes per level step (0 = 2^20): a wider level takes
                               several steps; the workspace grows with it           */
  uint32_t graph_samples;   /* batched: levels of at most this many samples run in
                               the loop graph, larger ones from the host (0 or
                               0xffffffff = every level in the graph)               */
  uint32_t part_shape;      /* partition of big segments: CT_PART_* (0 = default)   */
  uint32_t huge_rows;       /* nodes of at least this many rows partition with the
                               tree's mark bits in shared memory (0 = 4096, at
                               least 4096; 0xffffffff = never)                      */
  uint32_t small_rows;      /* nodes of at most this many rows partition one warp per
                               (node, 8 features) (0 = 4096 with 16-bit lists, 512
                               with 32-bit; else 512 .. 65536)                      */
} ct_fit_options;
/* ct_fit_options.part_shape: tile of a big segment's chain x ring buffers x
 * CTAs per SM of its partition.  Every shape partitions the same way. */
enum {
  CT_PART_2048_R2_B6 = 0, /* 2,048-element tiles, 2 buffers, 6 CTAs per SM (default) */
  CT_PART_1024_R3_B8 = 1, /* 1,024-element tiles, 3 buffers, 8 CTAs per SM           */
  CT_PART_4096_R2_B4 = 2, /* 4,096-element tiles, 2 buffers, 4 CTAs per SM           */
  CT_PART_2048_R3_B4 = 3, /* 2,048-element tiles, 3 buffers, 4 CTAs per SM           */
  CT_PART_SHAPES = 4
};
#define CT_HUGE_ROWS_MIN 4096u
/* ct_fit_options.flags.  CT_FIT_PROFILE: CUDA events around each kernel
 * group (ct_fit_stats.ms); the batched form then runs its levels from the
 * host.  The batched form otherwise runs its levels of at most
 * graph_samples samples as one CUDA graph with a device-side loop condition
 * (no host round trip between them); CT_FIT_HOST_LOOP asks for the
 * host-driven loop throughout (one host round trip per level, as the
 * reference's BFS, random_tree.py:428-431).  The trees are the same. */
enum { CT_FIT_PROFILE = 1, CT_FIT_HOST_LOOP = 2, CT_FIT_NO_VIRTUAL = 4 };
/* CT_FIT_NO_VIRTUAL: keep an index list for every feature.  By default, a
 * fit with label-carrying entries and at most 64 features keeps none for
 * its two-valued features other than feature 0: a node's sorted list of
 * such a feature is its rows in row order with the low value first, so one
 * row-order list per node and a value bit per row stand for them, and a
 * split moves that one list instead of theirs.  The trees are the same. */

/* Bytes of the ct_lists.mark buffer for n_slots tree slots. */
int ct_mark_bytes(uint32_t n_rows, uint32_t n_slots, size_t* bytes);

/* ---------------------------------------------------------------- info --- */
const char* ct_version(void);
/* Copies the last error text of this thread into buf; returns its length. */
int ct_last_error(char* buf, size_t len);

/* ---------------------------------------------------- data preparation --- */
/* Stable per-feature presort (replaces host np.argsort, random_forest.py:247).
 * x_fm [n_features][n_rows] -> out [n_features][n_rows] row ids (index_bytes). */
int ct_presort_workspace_size(uint32_t n_rows, uint32_t n_features, size_t* bytes);
int ct_presort(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t index_bytes,
               void* out, void* workspace, size_t workspace_bytes, void* stream);

/* In-bag rows of tree `tree` and stable compaction of every presorted row
 * into buffer 0 of `slot` (replaces _get_sorted_indices + bootstrap_fill.cu +
 * bootstrap_reshuffle.cu, random_forest.py:113-144).  n_in_dev[slot] receives
 * the in-bag count.  Without bootstrap the presort is copied. */
int ct_bootstrap_workspace_size(const ct_problem* p, size_t* bytes);
int ct_bootstrap_compact(const ct_problem* p, const ct_lists* lists, uint32_t slot, uint32_t tree,
                         uint32_t* n_in_dev, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------- hot path, per level --- */
/* Feature selection + Gini split scan + min-impurity reduction for n_nodes
 * nodes (replaces scan_gini_large/scan_reduce/compute_2d/reduce_2d/
 * find_min_imp, dfs_module.cu:24-208 + :310-491, and the BFS
 * scan_bfs/compute_2d/reduce/get_thresholds, bfs_module.cu:25-235, :379-401).
 * nodes/totals ([n_nodes][n_classes] uint32)/out/selected
 * ([n_nodes][max_features] uint32) are device pointers. */
int ct_split_workspace_size(const ct_problem* p, uint32_t n_nodes, uint64_t total_samples,
                            size_t* bytes);
int ct_split_nodes(const ct_problem* p, const ct_lists* lists, const ct_node* nodes,
                   const uint32_t* totals, uint32_t n_nodes, ct_split_result* out,
                   uint32_t* selected, void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free variant of ct_split_nodes; no counterpart in the
 * reference.  For callers that cannot allocate device memory (a process
 * whose device memory is held by another allocator's pool, a latency-bound
 * loop that must not call cudaMalloc/cudaFree, a C FFI host without device
 * buffers of its own): the scratch is a static 16 MiB array per device
 * instead of a caller workspace.  total_samples must be >= the sum of the
 * nodes' n; batches whose scratch exceeds 16 MiB are rejected with
 * CT_ERR_ARG.  Every call looks up the array's device address (no
 * allocation); the first call on a device may load the library's device
 * code and should come before any stream capture.  Calls that overlap on the
 * same device race on the shared array and must be serialized. */
int ct_split_nodes_noalloc(const ct_problem* p, const ct_lists* lists, const ct_node* nodes,
                           const uint32_t* totals, uint32_t n_nodes, uint64_t total_samples,
                           ct_split_result* out, void* stream);

/* Mark table + stable partition of every feature's node range into the
 * other buffer for each node whose split has a feature (replaces fill_table +
 * scan_reshuffle, dfs_module.cu:210-307, bfs_module.cu:238-377). */
int ct_partition_workspace_size(const ct_problem* p, uint32_t n_nodes, uint64_t total_samples,
                                size_t* bytes);
int ct_partition_nodes(const ct_problem* p, const ct_lists* lists, const ct_node* nodes,
                       const ct_split_result* splits, uint32_t n_nodes, void* workspace,
                       size_t workspace_bytes, void* stream);

/* -------------------------------------------------------- forest fit --- */
/* Grows trees first_tree .. first_tree+n_trees-1 into slots 0..n_trees-1 of
 * `trees` (replaces RandomForestClassifier.fit's tree loop + RandomClassifierTree.fit,
 * random_forest.py:292-336, random_tree.py:461-676).  Lists must hold n_trees slots
 * (one for CT_FIT_PLAIN); they are the fit's scratch, and while it runs their
 * entries may carry each row's label above its row id. */
int ct_fit_workspace_size(const ct_problem* p, uint32_t n_trees, const ct_fit_options* opt,
                          size_t* bytes);
int ct_fit(const ct_problem* p, const ct_lists* lists, uint32_t first_tree, uint32_t n_trees,
           const ct_fit_options* opt, const ct_tree_buffers* trees, void* workspace,
           size_t workspace_bytes, void* stream);

/* Forest queue: the batched fit of n_jobs independent forests through
 * shared level steps (one node list and one set of launches for all jobs'
 * nodes; the reference runs a queue as independent fits,
 * hybridforest/builder.py:79-141).  Job j grows trees first_tree ..
 * first_tree+n_trees-1 of its own problem into its lists, exactly the trees
 * ct_fit grows for it alone.  Its trees go to consecutive slots of `trees`,
 * after the slots of the jobs before it; trees->capacity must be at least
 * 2 * every job's n_rows.  Every job has the same index_bytes and
 * label_bytes; opt->mode must be CT_FIT_BATCHED (huge_rows is ignored: the
 * partition of big nodes reads marks from global memory).  ct_fit_stats
 * reports the whole queue. */
typedef struct ct_fit_job {
  ct_problem problem;
  ct_lists lists;            /* n_slots >= n_trees                            */
  uint32_t n_trees;
  uint32_t first_tree;
} ct_fit_job;
int ct_fit_queue_workspace_size(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* opt,
                                size_t* bytes);
int ct_fit_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* opt,
                 const ct_tree_buffers* trees, void* workspace, size_t workspace_bytes, void* stream);

/* Per-kernel-group statistics of the last ct_fit on the calling thread.
 * Launch counts and algorithmic bytes are always recorded; ms[] is filled
 * with CT_FIT_PROFILE (CUDA events recorded on the fit's stream around each
 * kernel group). */
enum {
  CT_K_SELECT = 0, CT_K_SCAN = 1, CT_K_REDUCE = 2, CT_K_MARK = 3,
  CT_K_PARTITION = 4, CT_K_CHILDREN = 5, CT_K_BOOTSTRAP = 6, CT_K_SUBTREE = 7,
  CT_NUM_KERNEL_GROUPS = 8
};
typedef struct ct_kernel_stats {
  uint64_t launches[8];  /* kernel launches per group                      */
  double ms[8];          /* summed event time per group (profiling on)      */
  double bytes[8];       /* algorithmic bytes per group                    */
  uint64_t steps;        /* level steps (node batches) run                 */
  uint64_t total_launches;
} ct_kernel_stats;
int ct_fit_stats(ct_kernel_stats* out);

/* Host-side: renumber one raw tree (host arrays) into breadth-first order,
 * left child before right.  Output arrays hold n_nodes entries. */
int ct_tree_canonicalize(const uint32_t* left, const uint32_t* right, const uint32_t* feature,
                         const float* threshold, const uint32_t* value, uint32_t n_nodes,
                         uint32_t* out_left, uint32_t* out_right, uint16_t* out_feature,
                         float* out_threshold, uint32_t* out_value);

/* Autotuner: fits n_trees sample trees (first tree 0) with each candidate
 * option set of the given mode and returns the fastest in *best (its time in
 * *best_ms).  Every candidate grows the same trees, so the choice changes
 * speed only.  Batched, in two stages: scan piece length (1024, 2048, 4096)
 * x warp-subtree cutoff (0, 32, 128); then, around each choice, the
 * partition shape (CT_PART_*) x huge_rows (4096, 16384, never), then
 * small_rows (default, 512, 2048, 8192).  Plain: the
 * depth-first/breadth-first switch, which the reference sets with an offline
 * regression (estimate_threshold.py, random_forest.py:278-289).  The
 * workspace must hold ct_autotune_workspace_size bytes; lists and trees as
 * for ct_fit with n_trees. */
int ct_autotune_workspace_size(const ct_problem* p, uint32_t n_trees, uint32_t mode, size_t* bytes);
int ct_autotune(const ct_problem* p, const ct_lists* lists, uint32_t n_trees, uint32_t mode,
                const ct_tree_buffers* trees, void* workspace, size_t workspace_bytes,
                ct_fit_options* best, float* best_ms, void* stream);

/* Row-major samples [n_rows][n_cols] -> feature-major [n_cols][n_rows] on the
 * device (the transpose of fit_init, random_forest.py:233).  When nan_flag
 * (device, zeroed by the caller) is given, it becomes nonzero if any value is
 * NaN: fits reject NaN, which has no place in the sorted order (the
 * reference does not check, random_forest.py:214-217). */
int ct_transpose_rows(const float* x_rm, uint32_t n_rows, uint32_t n_cols, float* x_cm,
                      uint32_t* nan_flag, void* stream);

/* Reads back the trees of one ct_fit call in canonical order.  counts[t]
 * (host) is trees->n_nodes[t]; tree t lands at [o_t, o_t + counts[t]) of the
 * host output arrays, o_t = counts[0] + ... + counts[t-1].  The used nodes
 * are gathered on the device into scratch (ct_fetch_trees_scratch bytes),
 * copied in one transfer, and renumbered on host threads.  Replaces the
 * full-buffer readback of decorate (random_tree.py:50-63). */
size_t ct_fetch_trees_scratch(uint64_t total_nodes, uint32_t n_trees);
int ct_fetch_trees(const ct_tree_buffers* trees, uint32_t n_trees, const uint32_t* counts,
                   void* scratch, size_t scratch_bytes, uint32_t* out_left, uint32_t* out_right,
                   uint16_t* out_feature, float* out_threshold, uint32_t* out_value, void* stream);

/* ----------------------------------------------------------- predict --- */
/* Packed forest: node i of the flat array is {threshold, feature, left, value}
 * with children left and left+1 inside the tree (breadth-first order);
 * tree_offset[t] is the first node of tree t.  Replaces BaseTree.gpu_predict +
 * predict.cu (base_tree.py:44-81, predict.cu:12-69) and the host vote
 * (random_forest.py:339-377).  x [n_rows][n_features] float32 row-major;
 * votes [n_rows][n_classes] uint32 (may be NULL); pred [n_rows] uint32 class
 * ids.  All device pointers; nodes 16-byte aligned; n_nodes nodes in all
 * (tree t ends where tree t+1 starts, the last tree at n_nodes).  Before the
 * walk the forest is checked on the device (its error word is pred[0], so
 * nothing is allocated): tree offsets strictly increasing inside the array,
 * every inner node's children after it inside its tree, features below
 * n_features, leaf classes below n_classes; a forest that fails returns
 * CT_ERR_ARG and is never walked.  The reference trusts its arrays
 * (predict.cu:50-67). */
typedef struct ct_packed_node {
  float threshold;
  uint32_t feature;
  uint32_t left;   /* 0 = leaf; else index (within the tree) of the left child */
  uint32_t value;  /* leaf class id                                           */
} ct_packed_node;

int ct_predict(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset,
               uint32_t n_trees, const float* x, uint32_t n_rows, uint32_t n_features,
               uint32_t n_classes, uint32_t* votes, uint32_t* pred, void* stream);

/* The forest check of ct_predict on host arrays (no device work): CT_OK, or
 * CT_ERR_ARG with the reason as the last error.  For callers that load
 * forests from files or other processes before uploading them; the
 * reference has no check (restore_forest, random_forest.py:18-23). */
int ct_check_forest(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset,
                    uint32_t n_trees, uint32_t n_features, uint32_t n_classes);

/* Compact forest: the same trees in 8-byte nodes, which halve the bytes a
 * walk step reads (the walk is bound by them).  With b = feature bits (the
 * smallest b >= 1 with 2^b >= n_features): inner node {threshold bits,
 * left << b | feature}, leaf {class id, 0}.  Usable when every tree has at
 * most 2^(32-b) nodes; same node order and tree_offset as the packed form. */
typedef struct ct_compact_node {
  uint32_t word0; /* threshold bits (inner) or class id (leaf)        */
  uint32_t word1; /* left << feature_bits | feature; 0 marks a leaf   */
} ct_compact_node;

/* 1 when trees of up to max_tree_nodes nodes fit the compact form. */
int ct_compact_fits(uint32_t n_features, uint32_t max_tree_nodes);
/* Device packed -> device compact (stream ordered); CT_ERR_ARG when the
 * trees do not fit.  A node whose child or feature does not fit the compact
 * fields becomes one that ct_predict_compact's forest check rejects. */
int ct_compact_forest(const ct_packed_node* nodes, uint32_t n_nodes, uint32_t n_features,
                      uint32_t max_tree_nodes, ct_compact_node* out, void* stream);
/* ct_predict on the compact form (nodes 8-byte aligned); same check, same
 * results. */
int ct_predict_compact(const ct_compact_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset,
                       uint32_t n_trees, const float* x, uint32_t n_rows, uint32_t n_features,
                       uint32_t n_classes, uint32_t* votes, uint32_t* pred, void* stream);

/* ----------------------------------------------------------- serving --- */
/* No counterpart in the reference (its predict re-uploads X and every tree
 * per call, base_tree.py:57-62).  A server keeps forests resident, batches
 * the predict requests that have arrived into one multi-request launch per
 * lane (small requests on a high-priority stream, large ones on a
 * low-priority stream), runs small fit jobs on worker streams, and holds all
 * its device memory inside an HBM budget.  Every device allocation happens in
 * ct_server_create: forests are carved from a pool reserved there, because a
 * device allocation made while requests run would serialize the streams. */
enum { CT_REQ_PREDICT = 0, CT_REQ_FIT = 1 };

typedef struct ct_server_config {
  uint32_t max_batch_rows;   /* rows per large-request batch (0 = 131072)            */
  uint32_t max_features;     /* largest feature count served (0 = 512)                */
  uint32_t small_rows;       /* <= this many rows: high-priority lane (0 = 4096)      */
  uint32_t fit_workers;      /* fit-job worker threads (0: fit jobs rejected)         */
  uint32_t max_fit_rows;     /* largest fit job (0 = 20000)                           */
  uint32_t max_fit_trees;    /* trees per fit job (0 = 10)                            */
  uint32_t max_classes;      /* forests with more classes are walked in one tree group
                                (0 = 64)                                              */
  uint32_t reserved;
  uint64_t hbm_budget_bytes; /* device bytes the server may hold (0 = 80% of free)    */
  uint64_t forest_pool_bytes;/* resident-forest pool inside the budget
                                (0 = min(4 GiB, a quarter of the budget))             */
} ct_server_config;

typedef struct ct_request {
  double arrival_s;          /* ct_server_replay: seconds after the replay starts    */
  uint32_t kind;             /* CT_REQ_PREDICT or CT_REQ_FIT                          */
  uint32_t forest;           /* predict: resident forest id                           */
  const float* x;            /* host [n_rows][n_features]; pinned for async copies;
                                small requests with mapped pinned x and pred are
                                served without copies                              */
  const uint32_t* y;         /* fit: host [n_rows] class ids < n_classes              */
  uint32_t* pred;            /* predict: host [n_rows] class ids (output)             */
  uint32_t n_rows;
  uint32_t n_features;       /* fit */
  uint32_t n_classes;        /* fit */
  uint32_t n_trees;          /* fit */
  uint32_t max_features;     /* fit (0 = ceil(sqrt(n_features)))                      */
  uint32_t status;           /* out: CT_OK or an error status                        */
  uint64_t seed;             /* fit */
  double latency_ms;         /* out: submit to completion                            */
  uint32_t result_forest;    /* out (fit): id of the new resident forest              */
  uint32_t pad_;
  void* pending_;            /* internal */
} ct_request;

typedef struct ct_server_stats {
  uint64_t requests, rows, batches, fit_jobs, rejected;
  double p50_ms, p99_ms;               /* all predict requests                 */
  double p50_small_ms, p99_small_ms;   /* predict requests of <= 4096 rows     */
  double p50_fit_ms, p99_fit_ms;       /* fit jobs                              */
  double max_ms, wall_s, rows_per_s;
  uint64_t hbm_used_bytes, hbm_budget_bytes;
  uint64_t forest_bytes, forest_pool_bytes; /* pool bytes held by forests / pool size */
  uint64_t zero_copy_requests;  /* small requests served from mapped host memory      */
} ct_server_stats;

int ct_server_create(const ct_server_config* cfg, void** handle);
int ct_server_destroy(void* handle);
/* Copies a packed forest (host arrays, layout of ct_predict) into the forest
 * pool; CT_ERR_OOM when the pool has no room.  The forest is checked on the
 * host first, as ct_predict checks it (CT_ERR_ARG when malformed). */
int ct_server_add_forest(void* handle, const ct_packed_node* nodes, uint32_t n_nodes,
                         const uint32_t* tree_offset, uint32_t n_trees, uint32_t n_features,
                         uint32_t n_classes, uint32_t* forest_id);
/* Size and shape of a resident forest, then its exact packed nodes and tree
 * offsets (host arrays of n_nodes and n_trees entries): forests fitted by
 * fit jobs can be read back, compared or serialized. */
int ct_server_forest_info(void* handle, uint32_t forest_id, uint32_t* n_nodes, uint32_t* n_trees,
                          uint32_t* n_features, uint32_t* n_classes);
int ct_server_read_forest(void* handle, uint32_t forest_id, ct_packed_node* nodes,
                          uint32_t* tree_offset);
/* Retires a forest: new requests for it fail with CT_ERR_ARG; its pool bytes
 * return once the batches already launched on it have completed. */
int ct_server_remove_forest(void* handle, uint32_t forest_id);
/* Queues a request now; its buffers must stay valid until ct_server_wait. */
int ct_server_submit(void* handle, ct_request* req);
int ct_server_wait(void* handle, ct_request* req, double timeout_s);
/* Submits each request at its arrival_s (open loop), waits for all, and
 * fills stats for this replay. */
int ct_server_replay(void* handle, ct_request* reqs, uint32_t n, double timeout_s,
                     ct_server_stats* stats);
int ct_server_get_stats(void* handle, ct_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* CUDATREE_B200_H */
