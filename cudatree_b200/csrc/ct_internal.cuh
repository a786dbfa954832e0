// Internal work-list records and launch helpers shared by the .cu files.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include <cuda/atomic>

#include "ct_common.cuh"

namespace ct {

// -------------------------------------------------------------- errors ---
void set_last_error(const std::string& msg);
const std::string& last_error_text();  // this thread's last error
#define CT_CUDA_TRY(expr)                                                              \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) {                                                           \
      ::ct::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(_e));        \
      return CT_ERR_CUDA;                                                              \
    }                                                                                  \
  } while (0)
#define CT_TRY(expr)                \
  do {                              \
    int _s = (expr);                \
    if (_s != CT_OK) return _s;     \
  } while (0)
#define CT_ARG_CHECK(cond, msg)                 \
  do {                                          \
    if (!(cond)) {                              \
      ::ct::set_last_error(msg);                \
      return CT_ERR_ARG;                        \
    }                                           \
  } while (0)
// Body of an extern "C" entry point: no C++ exception (std::bad_alloc from a
// message string, std::system_error from a lock) crosses the C ABI; it
// becomes CT_ERR_INTERNAL with the exception's text as the last error.
#define CT_GUARD(...)                                              \
  try {                                                            \
    __VA_ARGS__                                                    \
  } catch (const std::exception& e) {                              \
    try {                                                          \
      ::ct::set_last_error(std::string("exception: ") + e.what()); \
    } catch (...) {                                                \
    }                                                              \
    return CT_ERR_INTERNAL;                                        \
  } catch (...) {                                                  \
    return CT_ERR_INTERNAL;                                        \
  }

// Device-side error bits (Counters::error).
enum : uint32_t { DEV_ERR_TIMEOUT = 1u, DEV_ERR_CAPACITY = 2u, DEV_ERR_INTERNAL = 4u };
constexpr uint32_t NONE = 0xffffffffu;

// -------------------------------------------------------------- records ---
struct ScanPiece {        // one split-scan work item: part j of segment (node, slot)
  uint32_t node;
  uint32_t slot;
  uint32_t j;
  uint32_t npieces;       // pieces of this segment
  uint32_t carry;         // carry-table row of this piece (npieces > 1)
  uint32_t pad[3];
};
struct PieceBest {
  double score;
  uint32_t pos;
  float il;
  float ir;
  uint32_t pad;
};
struct SplitRec {         // a node that splits this step
  uint32_t node;
  uint32_t feature;
  uint32_t pos;
  uint32_t children;      // raw id of the left child (fit mode)
};
struct PartPiece {
  uint32_t split;
  uint32_t j;
  uint32_t npieces;
  uint32_t status;        // status column of this piece (npieces > 1)
};
struct Counters {
  uint32_t n_nodes;       // nodes in the current chunk
  uint32_t n_scan_pieces;
  uint32_t n_carry;
  uint32_t n_splits;
  uint32_t n_part_pieces; // mark-table pieces
  uint32_t n_status;
  uint32_t ticket;
  uint32_t error;
  uint32_t n_next;        // nodes appended to the next list
  uint32_t n_small;       // nodes appended to the subtree list
  uint32_t n_small_segs;  // partition segments of small splits
  uint32_t n_big_segs;
  uint32_t n_tiles;       // partition tiles of big splits
  uint32_t n_vpieces;     // row-list pieces (virtual features)
  uint32_t n_huge_segs;   // partition segments of k_part_seg
  uint32_t n_hchains;     // their chains (quads)
  uint32_t ticket_huge;   // k_part_seg's unit counter
  uint32_t n_bchains;     // active chains of k_part_big's segments
  uint32_t n_tv;          // scan pieces of two-valued features
  uint32_t claim[16];     // item counters of persistent launches (ITEM_* slots)
  unsigned long long next_total;
  unsigned long long small_total;
  unsigned long long split_total;  // samples in nodes partitioned this level
  unsigned long long scan_elems;   // (node, feature) elements scanned this level
  unsigned long long part_elems;   // (node, feature) elements partitioned this level
  unsigned long long vrows;        // row-list rows read by the virtual-feature counts this level
};

// Counters of one step, zeroed at its start (n_nodes set); the level totals
// (n_next, next_total, small_total, split_total, scan_elems, part_elems) are
// zeroed once per level by reset_level_counters.
// Slots of Counters::claim.  The subtree slots are zeroed by a fit's start
// and its loop graph, not per step (subtrees run after the level loop).
enum : uint32_t {
  ITEM_SELECT, ITEM_HIST, ITEM_CARRY, ITEM_SCAN, ITEM_TWO_VALUED, ITEM_REDUCE, ITEM_PLAN, ITEM_FILL,
  ITEM_CHILDREN, ITEM_VPIECES, ITEM_VCOUNT, ITEM_STEP_SLOTS, ITEM_SUBTREE = ITEM_STEP_SLOTS,
  ITEM_SUBTREE_WIDE
};
__device__ __forceinline__ void reset_step_counters(Counters* c, uint32_t n_nodes) {
  for (uint32_t i = 0; i < ITEM_STEP_SLOTS; ++i) c->claim[i] = 0;
  c->n_vpieces = 0;
  c->n_huge_segs = 0;
  c->n_hchains = 0;
  c->ticket_huge = 0;
  c->n_bchains = 0;
  c->n_nodes = n_nodes;
  c->n_scan_pieces = 0;
  c->n_carry = 0;
  c->n_tv = 0;
  c->n_splits = 0;
  c->n_part_pieces = 0;
  c->n_status = 0;
  c->ticket = 0;
  c->n_small_segs = 0;
  c->n_big_segs = 0;
  c->n_tiles = 0;
}
__device__ __forceinline__ void reset_level_counters(Counters* c) {
  c->n_next = 0;
  c->next_total = 0;
  c->small_total = 0;
  c->split_total = 0;
  c->scan_elems = 0;
  c->part_elems = 0;
  c->vrows = 0;
}

// One stable-partition segment: a node range in every feature list.
struct PartSeg {
  const void* in;         // element 0 of feature 0
  void* out;
  const uint32_t* bits;   // per-row left bit of the segment's tree
  uint32_t in_fstride;    // elements between consecutive features
  uint32_t out_fstride;
  uint32_t n;
  uint32_t nl;            // number of left rows
  uint32_t status;        // first status slot (tiled segments)
  uint64_t skip;          // features < 64 whose lists are left as they are (constant in the node)
  const uint64_t* skip_hi;  // the node's mask words of features 64.. (n_features > 64), else NULL
  uint32_t n_features;    // of the segment's job
  uint32_t row_mask;      // list entry -> row id of its mark bit (the job's View::row_mask)
};
struct PartTile {
  uint32_t seg;
  uint32_t j;
  uint32_t ntiles;
  uint32_t pad;
};
struct PartWork {
  PartSeg* small;
  uint32_t* n_small;
  uint32_t cap_small;
  PartSeg* big;
  uint32_t* n_big;
  uint32_t cap_big;
  const uint2* bchains;   // active chains (segment, feature) of the big segments
  uint32_t* n_bchains;
  uint32_t cap_bchains;
  PartSeg* huge;          // segments of k_part_seg (NULL: none)
  const uint2* hchains;   // their active chains (segment, feature or NONE), quads
  uint32_t* n_hchains;
  uint32_t cap_hchains;
  uint32_t* ticket_huge;
  uint32_t bit_words;     // mark-bit words of one tree
  uint32_t shape;         // CT_PART_* of k_part_big
  PartTile* tiles;
  uint32_t* n_tiles;
  uint32_t cap_tiles;
  uint64_t* status;       // [n_features][cap_status]
  uint32_t cap_status;
  uint32_t* ticket;
  uint32_t* error;
  uint32_t n_features;    // the most of any segment's job (k_part_small's feature blocks)
};

// View of the problem + lists passed by value to kernels.
struct View {
  const float* x_fm;
  const void* labels;
  void* si0;
  void* si1;
  uint8_t* mark;          // [n_slots][n_rows] bytes
  uint32_t* bits;         // [n_slots][bit_words] packed copy of mark
  uint32_t bit_words;
  uint32_t n_slots;
  uint32_t stride;
  uint32_t n_rows;
  uint32_t n_features;
  uint32_t n_classes;
  uint32_t max_features;
  uint32_t mss;
  int feistel_h;
  // List entries.  Lists a caller passes in hold plain row ids (row_mask all
  // ones, lab_shift 0).  The fit's own lists hold row | label << lab_shift
  // whenever both fit one entry (fit_label_shift), so a kernel that reads an
  // entry has the row's label without a gather into `labels`.
  uint32_t row_mask;
  uint32_t lab_shift;
  // Bit f set: feature f takes at most two distinct values over all rows
  // (feature_flags), so its split scan needs only the position of the node's
  // value boundary.  NULL: every feature takes the general scan.
  const uint32_t* fbin;
  // Virtual features (a fit with label-carrying entries and at most 64
  // features): two-valued features other than feature 0 whose index lists
  // are never partitioned.  A node's sorted list of such a feature is the
  // node's rows in row order, its low value's rows first (the stable order
  // of the presort), so it is fully described by the node's row list and
  // one bit per row: bit f of vrow[row] says x[f][row] is the feature's high
  // value.  The list slot of feature vslot (the lowest virtual feature)
  // holds the row list instead of that feature's list.  vval[f] = (low,
  // high).  vmask == 0: no virtual features.
  uint64_t vmask;
  const uint64_t* vrow;
  const float2* vval;
  uint32_t vslot;
  // A queue fit of several jobs (ct_fit_queue) passes the level kernels a
  // batch view whose jobs table holds one view per job; a work item reads
  // the view of its node's job (job_view).  Tree slots are numbered across
  // the jobs, and a job's lists and mark bits are indexed by slot -
  // slot_base.  The scratch strides are the batch's: sel_stride selected
  // feature slots and mask_stride constant-mask words per node (a job's
  // max_features and n_features are its own).  One job: jobs NULL,
  // slot_base 0, sel_stride = max_features, mask_stride =
  // mask_words(n_features).
  const View* jobs;
  const uint32_t* slot_job;
  uint32_t slot_base;
  uint32_t sel_stride;
  uint32_t mask_stride;
};
// `const View& V`: the view of the job that owns tree slot SLOT.  In a
// kernel instantiated for a queue (template flag Q) it is that job's entry
// of the batch view VB's table; otherwise V is VB itself, so a fit of one
// job compiles as if the lookup were not there.
#define CT_JOB_VIEW(V, VB, SLOT)                              \
  View V##_job;                                               \
  if constexpr (Q) V##_job = (VB).jobs[(VB).slot_job[SLOT]];  \
  const View& V = Q ? V##_job : (VB)
__device__ __forceinline__ bool two_valued(const View& v, uint32_t f) {
  return v.fbin && ((__ldg(v.fbin + (f >> 5)) >> (f & 31)) & 1u);
}
__host__ __device__ __forceinline__ bool is_virtual(const View& v, uint32_t f) {
  return f < 64 && ((v.vmask >> f) & 1u);
}
// Features whose lists a split leaves as they are: the virtual ones except
// the row-list slot.
__host__ __device__ __forceinline__ uint64_t virtual_skip(const View& v) {
  return v.vmask ? v.vmask & ~(1ull << v.vslot) : 0ull;
}

// Packed mark table: bit r of a slot's words is row r's left flag.  The
// words of one tree (N/8 bytes) fit in an SM's L1, unlike the byte table.
__host__ __device__ __forceinline__ uint32_t mark_bit_words(uint32_t n_rows) {
  return ((n_rows + 31) / 32 + 3) & ~3u;
}
__host__ __device__ __forceinline__ size_t mark_bits_offset(uint32_t n_rows, uint32_t n_slots) {
  return ((size_t)n_slots * n_rows + 255) & ~size_t(255);
}
__device__ __forceinline__ bool left_bit(const uint32_t* bits, uint32_t row) {
  return (__ldg(bits + (row >> 5)) >> (row & 31)) & 1u;
}

// L2 cache policies.  The index lists stream through once per level (251 MB
// at covtype size, twice L2), while x and the mark bits are gathered at
// random: list traffic is marked evict-first so the gathered arrays keep
// their lines.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

template <typename IdxT>
__device__ __forceinline__ IdxT* list_ptr(const View& v, uint32_t buf, uint32_t slot, uint32_t f) {
  IdxT* base = reinterpret_cast<IdxT*>(buf ? v.si1 : v.si0);
  return base + ((size_t)(slot - v.slot_base) * v.n_features + f) * v.stride;
}
// mark bits of the tree in slot `slot`
__device__ __forceinline__ uint32_t* slot_bits(const View& v, uint32_t slot) {
  return v.bits + (size_t)(slot - v.slot_base) * v.bit_words;
}
__device__ __forceinline__ uint32_t entry_row(const View& v, uint32_t e) { return e & v.row_mask; }
template <typename LabT>
__device__ __forceinline__ uint32_t entry_label(const View& v, uint32_t e) {
  return v.lab_shift ? e >> v.lab_shift : (uint32_t)reinterpret_cast<const LabT*>(v.labels)[e];
}

// Raw tree arrays (fit mode).
struct TreeView {
  uint32_t* left;
  uint32_t* right;
  uint32_t* feature;
  float* threshold;
  uint32_t* value;
  uint32_t* n_nodes;
  uint32_t capacity;
  uint32_t slot_base;     // tree slot = list slot + slot_base
  uint32_t enabled;
};

// The node lists of one level step, in device memory: written by the step's
// first kernel (k_reset_step, or the graph-driven loop's step kernel) and
// read by every later kernel of the step, so the step's launches do not
// depend on which buffer holds the level or where its chunk starts.
struct StepLists {
  const ct_node* nodes;       // the step's nodes
  const uint32_t* tot;        // their class totals [n][n_classes]
  const uint64_t* node_mask;  // their constant-feature masks, or NULL (see LevelScratch)
  ct_node* next;              // the next level's list: children are appended
  uint32_t* next_tot;         // their class totals
  uint64_t* next_mask;        // their masks, or NULL
  uint32_t scan_piece;        // elements per split-scan piece in this step
};

// Scratch of one level step, carved from the caller's workspace.
struct LevelScratch {
  uint32_t cap_nodes;
  uint32_t cap_scan;
  uint32_t cap_carry;
  uint32_t cap_part;
  uint32_t cap_status;
  uint32_t* sel;          // [cap_nodes][max_features]
  uint32_t* nsel;         // [cap_nodes]
  uint32_t* piece_base;   // [cap_nodes]
  uint32_t* piece_cnt;    // [cap_nodes]
  ScanPiece* pieces;      // [cap_scan]
  uint32_t* carry;        // [cap_carry][n_classes]
  uint32_t* carry_piece;  // [cap_carry] the scan piece of each carry row (pieces of multi-piece segments)
  uint32_t* tv_pieces;    // [cap_scan] the scan pieces of two-valued features
  PieceBest* best;        // [cap_scan]
  ct_split_result* result;// [cap_nodes]
  SplitRec* splits;       // [cap_nodes]
  uint32_t* split_left;   // [cap_nodes][n_classes]
  PartPiece* part;        // [cap_part] mark-table pieces
  PartSeg* small_segs;    // [cap_nodes]
  PartSeg* big_segs;      // [cap_nodes]
  PartSeg* huge_segs;     // [cap_huge] segments of at least HUGE_SEG rows (k_part_seg)
  uint2* hchains;         // [cap_hchains] their active chains in quads
  uint32_t cap_huge;
  uint32_t cap_hchains;
  uint2* bchains;         // [cap_bchains] active chains of the big segments
  uint32_t cap_bchains;
  PartTile* tiles;        // [cap_status]
  uint64_t* status;       // [n_features][cap_status]
  Counters* ctr;
  // The step's lists.  Constant-feature masks exist in a batched fit: node
  // i of the step owns View::mask_stride words from node_mask +
  // i * mask_stride, and bit f % 64 of word f / 64 says that feature f is
  // constant in the node, so its lists are not partitioned and k_select
  // does not read them; k_children writes the next list's masks.  Feature 0
  // is never in a mask (leaf labels and subtrees read its lists).
  StepLists* step;
  uint32_t huge_rows;     // segments of at least this many rows take k_part_seg (>= HUGE_SEG)
  uint32_t part_shape;    // CT_PART_* of k_part_big
  uint32_t small_rows;    // segments of at most this many rows take k_part_small (>= SMALL_SEG)
  // Virtual features (View::vmask), else NULL / 0:
  uint32_t* vcnt;         // [cap_nodes][64] rows of each node with the feature's high value
  uint32_t* vcls;         // [cap_nodes][n_features][n_classes] those rows by class
  uint2* vpieces;         // [cap_vpieces] (node, piece) of the nodes' row lists
  uint32_t cap_vpieces;
};
__device__ __forceinline__ bool masked(uint64_t m, uint32_t f) { return f < 64 && ((m >> f) & 1u); }
// words of one node's constant-feature mask
__host__ __device__ __forceinline__ uint32_t mask_words(uint32_t n_features) { return (n_features + 63) / 64; }
// bit f of a node's multi-word mask (NULL: no feature masked)
__device__ __forceinline__ bool mask_bit(const uint64_t* m, uint32_t f) { return m && ((m[f >> 6] >> (f & 63)) & 1u); }
// feature f's lists are left as they are in segment sg
__device__ __forceinline__ bool seg_skips(const PartSeg& sg, uint32_t f) {
  return f < 64 ? ((sg.skip >> f) & 1u) : mask_bit(sg.skip_hi, f - 64);
}

// Per-kernel-group launch counts and CUDA-event timing of one fit.
struct Prof {
  bool timing = false;
  cudaStream_t st = nullptr;
  ct_kernel_stats stats{};
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ranges;
  int open_kernel = -1;
  cudaEvent_t open_ev = nullptr;
  void begin(int k) {
    if (!timing) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    open_kernel = k;
    open_ev = e;
  }
  void end() {
    if (!timing || open_kernel < 0) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    ranges.push_back({open_kernel, {open_ev, e}});
    open_kernel = -1;
  }
  void launched(int k, uint64_t n = 1) {
    stats.launches[k] += n;
    stats.total_launches += n;
  }
  void finish() {
    if (!ranges.empty()) cudaStreamSynchronize(st);
    for (auto& r : ranges) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r.second.first, r.second.second);
      stats.ms[r.first] += ms;
      cudaEventDestroy(r.second.first);
      cudaEventDestroy(r.second.second);
    }
    ranges.clear();
  }
};
Prof* current_prof();  // profile of the fit running on this thread (never NULL)

// Bump allocator over a caller workspace (256-byte aligned carving).
struct Arena {
  char* base;
  size_t size;
  size_t used;
  template <typename T>
  T* take(size_t count) {
    size_t off = (used + 255) & ~size_t(255);
    size_t bytes = count * sizeof(T);
    used = off + bytes;
    if (base == nullptr || used > size) return nullptr;
    return reinterpret_cast<T*>(base + off);
  }
  bool ok() const { return used <= size; }
};

// Tile shapes.
constexpr uint32_t DEFAULT_SCAN_PIECE = 2048;   // elements per split-scan work item
// Split-scan piece of a fit's level of `samples` samples whose nodes scan
// mat16 / 16 lists each on average: the fit's piece, halved (not below
// MIN_STEP_PIECE) while the level would make fewer than STEP_PIECES pieces,
// so that a small level does not wait on a few warps' long pieces.  The
// pieces do not change the result.  samples = 0 gives the smallest piece a
// fit can use (its scratch capacities).
constexpr uint32_t MIN_STEP_PIECE = 512;
constexpr uint64_t STEP_PIECES = 12288;
__host__ __device__ __forceinline__ uint32_t step_piece(uint64_t samples, uint32_t piece, uint32_t mat16) {
  while (piece >= 2 * MIN_STEP_PIECE && (uint64_t)mat16 * samples < 16 * STEP_PIECES * piece) piece >>= 1;
  return piece;
}
constexpr uint32_t PART_ROUNDS = 16;            // rounds of 32 held in registers
constexpr uint32_t PART_PIECE = 32 * PART_ROUNDS;
constexpr uint32_t TILE_ELEMS = 4096;           // partition tile of big segments
// Segments of at least HUGE_SEG rows are partitioned with the tree's mark
// bits staged in shared memory (k_part_seg) when those bits fit the budget.
constexpr uint32_t HUGE_SEG = CT_HUGE_ROWS_MIN;  // default and smallest ct_fit_options.huge_rows (capacities)
constexpr uint32_t HUGE_BITS_MAX = 150u * 1024u;
__host__ __device__ __forceinline__ bool huge_partition_ok(uint32_t bit_words) {
  return (uint64_t)bit_words * 4u <= HUGE_BITS_MAX;
}
constexpr uint32_t SMALL_SEG = 32 * PART_ROUNDS; // segments up to this size: one warp
// Default ct_fit_options.small_rows: with 16-bit entries a warp per (segment,
// 8 features) beats a CTA per chain up to a few thousand rows (the CTA's tile
// of 2,048 entries is mostly idle there); with 32-bit entries from 513 rows on.
inline uint32_t default_small_rows(uint32_t index_bytes) { return index_bytes == 2 ? 4096u : SMALL_SEG; }
constexpr int WARPS_PER_BLOCK = 4;
constexpr int THREADS_PER_BLOCK = 32 * WARPS_PER_BLOCK;

// Bounds of one step: nodes in the chunk and samples they hold.
struct LevelBounds {
  uint64_t nodes;
  uint64_t samples;
};
struct LevelCaps {
  uint32_t nodes, scan, carry, part, status, vpieces, huge, hchains, bchains;
};
LevelCaps level_caps(const View& v, uint32_t scan_piece, LevelBounds b);
constexpr uint32_t VPIECE = 2048;  // rows per row-list piece (virtual features)
// Scratch of virtual features: carved when `virt` (the fit may have some).
bool virtual_possible(const ct_problem* p);
bool carve_level_scratch(Arena& a, const View& v, const LevelCaps& c, LevelScratch* s, bool virt = false);
size_t level_scratch_bytes(const View& v, const LevelCaps& c, bool virt = false);

// Level-step launches (ct_level.cu).  The step's node count is in
// s.ctr->n_nodes and its lists in *s.step (both on the device, set by the
// step's reset kernel); b bounds the step (nodes, samples) and sizes the
// grids.  Every warp-per-item kernel loops over its items, so with
// `persistent` a launch takes at most the blocks resident at once: a
// graph-driven loop, whose launches are fixed at capture, passes the
// workspace's bounds.
int launch_split(const View& v, uint32_t index_bytes, uint32_t label_bytes, const LevelScratch& s, LevelBounds b,
                 uint32_t scan_piece, bool persistent, cudaStream_t st);
int launch_partition(const View& v, uint32_t index_bytes, uint32_t label_bytes, const LevelScratch& s,
                     LevelBounds b, const TreeView& tv, bool persistent, cudaStream_t st);
// Children of the step's splits: appended to the next list (at most
// cap_next) or, when they have at most small_cut rows, to the subtree list
// while it has room (cap_small); a child that finds the subtree list full
// goes to the next list (the level steps grow the same subtrees).
int launch_children(const View& v, uint32_t index_bytes, uint32_t label_bytes, const LevelScratch& s,
                    LevelBounds b, const TreeView& tv, uint32_t cap_next, uint32_t small_cut, ct_node* small,
                    uint32_t cap_small, bool persistent, cudaStream_t st);
// Warp subtrees of the small nodes the children steps set aside (the count
// is s.ctr->n_small, at most cap_small; the grid covers `bound` of them and
// loops over the rest); wide: some may have 33..128 rows.
int launch_subtrees(const View& v, uint32_t ib, uint32_t lb, const ct_node* small, uint32_t cap_small,
                    uint32_t bound, bool wide, bool persistent, const LevelScratch& s, const TreeView& tv,
                    cudaStream_t st);
// Stable partition of segments (ct_partition.cu).
int launch_seg_partition(uint32_t index_bytes, const PartWork& w, uint64_t bound_small, uint64_t bound_tiles,
                         cudaStream_t st);
PartWork level_part_work(const View& v, const LevelScratch& s);

// Start of a step (device-side, stream ordered): per-step counters reset,
// n_nodes and the step's lists set.
int launch_reset_step(const LevelScratch& s, uint32_t n_nodes, const StepLists& lists, cudaStream_t st);
// Blocks of a warp-per-item launch: one warp per item, at most grid_cap
// blocks (0: no cap).
uint32_t item_blocks(uint64_t warps, uint32_t grid_cap);

View make_view(const ct_problem* p, const ct_lists* l);
// Bits of a row id when a row id and a label fit one list entry together
// (the shift of the label), else 0.
uint32_t fit_label_shift(const ct_problem* p);

// One request of a multi-request predict launch (ct_predict.cu): blocks
// [block0, block0 + tiles * ceil(n_trees / group)) of the launch are its,
// group-major; rows [row0, row0 + n_rows) of the batch are its.
struct BatchReq {
  const void* nodes;      // packed (fbits 0) or compact nodes
  const uint32_t* tree_off;
  const float* x;         // [n_rows][n_features] on the device
  uint32_t* pred;         // [n_rows] on the device
  uint32_t* votes;        // [n_rows][n_classes] zeroed table (grouped requests)
  uint32_t n_rows;
  uint32_t n_features;
  uint32_t n_classes;
  uint32_t n_trees;
  uint32_t block0;
  uint32_t tiles;
  uint32_t group;         // trees per group (>= n_trees: one group, no vote table)
  uint32_t row0;
  uint32_t fbits;         // 0: packed nodes; else compact nodes with this many feature bits
  uint32_t rpb;           // rows per tile (predict_rows_per_block)
};
uint32_t predict_rows_per_block(uint32_t n_classes, uint32_t n_features);
size_t predict_tile_smem(uint32_t rpb, uint32_t n_classes, uint32_t n_features);
uint32_t predict_group_size(uint32_t n_trees, uint64_t n_nodes, size_t node_bytes);
uint32_t compact_feature_bits(uint32_t n_features);
bool compact_fits(uint32_t n_features, uint64_t max_tree_nodes);
void compact_host(const ct_packed_node* in, uint32_t n, uint32_t fbits, ct_compact_node* out);
// CT_ERR_ARG unless every tree [off[t], off[t + 1] or n_nodes) is non-empty,
// every inner node's children (left, left + 1; local indices) come after it
// inside its tree, features are < n_features and leaf classes < n_classes.
int check_forest_host(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* off, uint32_t n_trees,
                      uint32_t n_features, uint32_t n_classes);
int predict_batch(const BatchReq* reqs_dev, uint32_t n_req, uint32_t total_blocks, uint32_t total_rows,
                  size_t smem, bool any_grouped, cudaStream_t st);
// Bit f of bits ([ceil(n_features / 32)] words, zeroed here): feature f takes
// at most two distinct values (-0.0 and +0.0 count as one, as in the scan's
// comparisons).
// vals (or NULL): each feature's (minimum, maximum); work: device scratch
// of feature_flags_work_bytes(n_features).
int feature_flags(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t* bits, float2* vals, void* work,
                  cudaStream_t st);
size_t feature_flags_work_bytes(uint32_t n_features);
// Value bits of the virtual features vmask (View::vrow) into out[n_rows].
int virtual_rows(const float* x_fm, uint32_t n_rows, uint64_t vmask, const float2* vval, uint64_t* out,
                 cudaStream_t st);
int transpose_rows(const float* x_rm, uint32_t n_rows, uint32_t n_cols, float* x_cm, cudaStream_t st,
                   uint32_t* nan_flag = nullptr);
int check_problem(const ct_problem* p);

}  // namespace ct
