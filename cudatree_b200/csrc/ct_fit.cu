// Forest fit orchestration.
//
// CT_FIT_PLAIN mirrors the reference tree builder (random_tree.py:461-676):
// one tree at a time; nodes larger than bfs_threshold are split one by one
// in depth-first order with a host round trip per node (random_tree.py:580-676),
// smaller nodes are queued and split breadth-first one level per step for the
// tree (random_tree.py:309-458).
//
// CT_FIT_BATCHED grows every tree of the call at once, level-synchronously:
// one step splits every pending node of every tree, with one host read of
// the step counters per level.  Both forms run the same level kernels and the
// same canonical rule, so their trees are identical after canonical
// renumbering.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "ct_internal.cuh"

namespace ct {

size_t bootstrap_scratch_bytes(uint32_t n_rows, uint32_t n_features, uint32_t n_slots);
int bootstrap_many(const ct_problem* p, const ct_lists* l, uint32_t slot_lo, uint32_t n_slots, uint32_t tree_lo,
                   const void* src, uint32_t row_mask, uint64_t skip, uint32_t* n_in_dev, void* ws, size_t wsb,
                   cudaStream_t st);
int pack_presort(const ct_problem* p, void* out, uint32_t shift, uint32_t ident, uint64_t skip, cudaStream_t st);

namespace {

constexpr uint32_t CHUNK_NODES_MAX = 1u << 20;
// every level in the loop graph: its launches are persistent like the host
// loop's, so a larger level gains nothing from the host's round trip
constexpr uint64_t DEFAULT_GRAPH_SAMPLES = UINT64_MAX;

// Class histogram of every slot's in-bag rows: grid (blocks, slots), one
// shared-memory histogram per block flushed with global atomics.
template <typename IdxT, typename LabT>
__global__ void k_root_hist(View v, const uint32_t* n_in, uint32_t slot_lo, uint32_t* hist_out) {
  extern __shared__ uint32_t hist[];
  const uint32_t slot = slot_lo + blockIdx.y;
  const uint32_t C = v.n_classes;
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x) hist[c] = 0;
  __syncthreads();
  const uint32_t n = n_in[slot];
  const IdxT* lst = list_ptr<IdxT>(v, 0, slot, 0);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&hist[entry_label<LabT>(v, lst[i])], 1u);
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < C; c += blockDim.x)
    if (hist[c]) atomicAdd(&hist_out[(size_t)blockIdx.y * C + c], hist[c]);
}

// Root record of each slot (block per slot): a leaf if it holds fewer than
// min_samples_split rows, else appended to the first level's list.
template <typename IdxT, typename LabT>
__global__ void k_root(View v, const uint32_t* n_in, uint32_t slot_lo, uint64_t seed, uint32_t tree_lo,
                       TreeView tv, const uint32_t* hist_in, ct_node* out, uint32_t* out_tot, uint32_t cap,
                       Counters* ctr, uint64_t* out_mask) {
  __shared__ uint32_t s_idx;
  extern __shared__ unsigned long long s_mask[];  // [mask_words(n_features)] with out_mask
  const uint32_t slot = slot_lo + blockIdx.x;
  const uint32_t C = v.n_classes;
  const uint32_t n = n_in[slot];
  const IdxT* lst = list_ptr<IdxT>(v, 0, slot, 0);
  if (threadIdx.x == 0) {
    const uint32_t ts = slot + tv.slot_base;
    tv.n_nodes[ts] = 1;
    ct_node nd;
    nd.slot = slot;
    nd.start = 0;
    nd.n = n;
    nd.raw_id = 0;
    nd.key = root_key(tree_key(seed, tree_lo + blockIdx.x));
    nd.impurity = 1.0f;
    nd.buf = 0;
    s_idx = NONE;
    if (n < v.mss || n == 0) {
      const size_t off = (size_t)ts * tv.capacity;
      tv.left[off] = 0;
      tv.right[off] = 0;
      tv.feature[off] = 0;
      tv.threshold[off] = 0.f;
      tv.value[off] = n ? entry_label<LabT>(v, lst[0]) : 0u;
    } else {
      const uint32_t idx = atomicAdd(&ctr->n_next, 1u);
      if (idx < cap) {
        out[idx] = nd;
        atomicAdd(&ctr->next_total, (unsigned long long)n);
        s_idx = idx;
      } else {
        atomicOr(&ctr->error, DEV_ERR_CAPACITY);
      }
    }
  }
  __syncthreads();
  if (s_idx != NONE)
    for (uint32_t c = threadIdx.x; c < C; c += blockDim.x)
      out_tot[(size_t)s_idx * C + c] = hist_in[(size_t)blockIdx.x * C + c];
  if (out_mask && s_idx != NONE) {  // features constant over the tree's in-bag rows (feature 0 excepted)
    const uint32_t mw = mask_words(v.n_features);
    for (uint32_t k = threadIdx.x; k < mw; k += blockDim.x) s_mask[k] = 0;
    __syncthreads();
    for (uint32_t f = threadIdx.x; f < v.n_features; f += blockDim.x) {
      if (f == 0 || is_virtual(v, f)) continue;
      const IdxT* lf = list_ptr<IdxT>(v, 0, slot, f);
      const float* xf = v.x_fm + (size_t)f * v.n_rows;
      if (xf[entry_row(v, lf[0])] == xf[entry_row(v, lf[n - 1])]) atomicOr(&s_mask[f >> 6], 1ull << (f & 63));
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < mw; k += blockDim.x) out_mask[(size_t)s_idx * v.mask_stride + k] = s_mask[k];
  }
}

__global__ void k_begin_level(Counters* c) { reset_level_counters(c); }

void begin_level(Counters* c, cudaStream_t st) {
  k_begin_level<<<1, 1, 0, st>>>(c);
  current_prof()->launched(CT_K_CHILDREN);
}

// Algorithmic bytes of one level, from the device counters of the level
// (a scanned entry that carries its label needs no label read).
void account_level(const ct_problem* p, const View& view, const Counters& h) {
  Prof* pf = current_prof();
  const double w = p->index_bytes, l = view.lab_shift ? 0.0 : p->label_bytes, v = sizeof(float);
  pf->stats.bytes[CT_K_SCAN] += (double)h.scan_elems * (w + l + v) + (double)h.vrows * (w + 8.0);
  pf->stats.bytes[CT_K_MARK] += (double)h.split_total * (w + 1.0);
  pf->stats.bytes[CT_K_PARTITION] += (double)h.part_elems * (2.0 * w + 1.0);  // chains actually partitioned
  pf->stats.steps += 1;
}

// State of the graph-driven level loop (device memory).
struct LoopCtl {
  uint32_t cur;      // list holding the current level
  uint32_t lo;       // first node of the current chunk
  uint32_t n_level;  // nodes of the current level
  uint32_t levels;   // levels finished
  uint32_t steps;    // steps run
  uint32_t pad[3];
  unsigned long long scan_elems;   // totals of the finished levels
  unsigned long long split_total;
  unsigned long long part_elems;
  unsigned long long vrows;
  unsigned long long level_samples;  // samples of the current level (its scan piece)
};

struct FitLayout {
  uint32_t n_slots;
  uint32_t cap_list;
  uint32_t chunk;
  uint32_t scan_piece;
  uint32_t mat16;        // 16 x the lists a node's split scan reads on average (step_piece)
  uint32_t subtree_cut;  // nodes of at most this many rows are grown by warp subtrees (0: off)
  uint32_t cap_small;
  bool host_loop;        // batched form: per-level host round trips instead of the loop graph
  uint64_t graph_samples; // batched form: levels of at most this many samples run in the loop graph
  ct_node* small;        // small nodes waiting for their warp subtree (kept across levels)
  mutable uint64_t small_bound;  // upper bound of the entries in small
  uint32_t* n_in;
  uint32_t* fbin;        // two-valued feature bits (feature_flags)
  void* ffwork;          // feature_flags scratch
  bool virt;             // the fit may have virtual features (View::vmask)
  uint64_t* vrow;        // [n_rows] their value bits
  float2* vval;          // [n_features] (low, high) values
  ct_node* list[2];
  uint32_t* tot[2];
  uint64_t* mask[2];     // constant-feature masks of the lists (batched form), else NULL
  uint32_t mask_words;   // words of one node's mask
  LevelScratch s;
  struct LoopCtl* ctl;   // state of the graph-driven level loop
  void* boot_ws;
  size_t boot_bytes;
  size_t bytes;
};

bool layout(const ct_problem* p, uint32_t n_trees, const ct_fit_options* o, char* base, size_t size,
            FitLayout* L) {
  View v = make_view(p, nullptr);
  const uint32_t slots = (o->mode == CT_FIT_PLAIN) ? 1u : n_trees;
  const uint64_t S = (uint64_t)slots * p->n_rows;
  const uint64_t cap_list64 = S / 2 + slots + 2;
  L->n_slots = slots;
  L->cap_list = (uint32_t)std::min<uint64_t>(cap_list64, 0xffffffffull);
  L->chunk = std::min<uint32_t>(L->cap_list, o->step_nodes ? o->step_nodes : CHUNK_NODES_MAX);
  if (virtual_possible(p) && !(o->flags & CT_FIT_NO_VIRTUAL)) {
    // the per-node class counts of the virtual features stay within 1 GiB
    const uint64_t per_node = (uint64_t)p->n_features * p->n_classes * sizeof(uint32_t);
    L->chunk = std::min<uint32_t>(L->chunk, (uint32_t)std::max<uint64_t>(4096, (1ull << 30) / per_node));
  }
  L->scan_piece = o->scan_piece ? o->scan_piece : DEFAULT_SCAN_PIECE;
  // the warp subtree packs a row id into 27 bits of its sort key
  L->subtree_cut = p->n_rows < (1u << 27) ? std::min<uint32_t>(o->subtree_cutoff, 128u) : 0u;
  L->cap_small = L->subtree_cut ? 2 * L->chunk : 0u;
  L->host_loop = (o->flags & CT_FIT_HOST_LOOP) != 0;
  L->graph_samples = o->graph_samples == 0xffffffffu ? UINT64_MAX
                     : o->graph_samples               ? o->graph_samples
                                                      : DEFAULT_GRAPH_SAMPLES;
  Arena a{base, size, 0};
  L->small = L->cap_small ? a.take<ct_node>(L->cap_small) : nullptr;
  L->small_bound = 0;
  L->n_in = a.take<uint32_t>(slots);
  L->fbin = a.take<uint32_t>((p->n_features + 31) / 32);
  L->ffwork = a.take<char>(feature_flags_work_bytes(p->n_features));
  L->virt = virtual_possible(p) && !(o->flags & CT_FIT_NO_VIRTUAL);
  L->vrow = L->virt ? a.take<uint64_t>(p->n_rows) : nullptr;
  L->vval = L->virt ? a.take<float2>(p->n_features) : nullptr;
  // the plain form moves nodes through the host, so only the batched form keeps masks
  const bool masks = o->mode == CT_FIT_BATCHED;
  L->mask_words = mask_words(p->n_features);
  for (int i = 0; i < 2; ++i) {
    L->list[i] = a.take<ct_node>(L->cap_list);
    L->tot[i] = a.take<uint32_t>((size_t)L->cap_list * p->n_classes);
    L->mask[i] = masks ? a.take<uint64_t>((size_t)L->cap_list * mask_words(p->n_features)) : nullptr;
  }
  L->boot_bytes = bootstrap_scratch_bytes(p->n_rows, p->n_features, slots);
  L->boot_ws = a.take<char>(L->boot_bytes);
  L->mat16 = 16 * std::min(p->max_features, p->n_features);
  LevelCaps caps = level_caps(v, step_piece(0, L->scan_piece, 1), LevelBounds{L->chunk, S});
  carve_level_scratch(a, v, caps, &L->s, L->virt);
  L->s.huge_rows = o->huge_rows ? o->huge_rows : HUGE_SEG;
  L->s.part_shape = o->part_shape;
  L->s.small_rows = o->small_rows ? o->small_rows : default_small_rows(p->index_bytes);
  L->ctl = a.take<LoopCtl>(1);
  L->bytes = a.used + 256;
  return base != nullptr && a.ok();
}

struct Host {
  Counters c;
};

int read_counters(const FitLayout& L, Counters* h, cudaStream_t st) {
  CT_CUDA_TRY(cudaMemcpyAsync(h, L.s.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  if (h->error) {
    if (h->error & DEV_ERR_TIMEOUT) {
      set_last_error("device look-back wait gave up (timeout)");
      return CT_ERR_TIMEOUT;
    }
    if (h->error & DEV_ERR_CAPACITY) {
      set_last_error("device work-list or tree capacity exceeded");
      return CT_ERR_CAPACITY;
    }
    set_last_error("device consistency check failed");
    return CT_ERR_INTERNAL;
  }
  return CT_OK;
}

int check_boot_error(const FitLayout& L, cudaStream_t st) {
  uint32_t w[2] = {0, 0};
  CT_CUDA_TRY(cudaMemcpyAsync(w, L.boot_ws, sizeof(w), cudaMemcpyDeviceToHost, st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  if (w[1]) {
    set_last_error("bootstrap compaction flagged a device error");
    return CT_ERR_TIMEOUT;
  }
  return CT_OK;
}

void account_bootstrap(const ct_problem* p, uint64_t skip) {
  Prof* pf = current_prof();
  const double w = p->index_bytes, n = p->n_rows, f = p->n_features - (p->bootstrap ? __builtin_popcountll(skip) : 0);
  // read presort + gather mark, write the in-bag part (about 0.632 n per feature)
  pf->stats.bytes[CT_K_BOOTSTRAP] += n * f * (w + 1.0) + (p->bootstrap ? 0.632 : 1.0) * n * f * w;
  pf->launched(CT_K_BOOTSTRAP, p->bootstrap ? 3 : 1);
}

template <typename IdxT, typename LabT>
int launch_root(const View& v, const FitLayout& L, uint32_t slot_lo, uint32_t n_slots, uint64_t seed,
                uint32_t tree_lo, const TreeView& tv, int cur, cudaStream_t st) {
  const size_t C = v.n_classes;
  // the histograms go to the tail of the next list's totals, which the root step does not use
  uint32_t* hist = L.tot[1 - cur];
  CT_CUDA_TRY(cudaMemsetAsync(hist, 0, n_slots * C * sizeof(uint32_t), st));
  const uint32_t blocks = std::min<uint32_t>(ceil_div(v.n_rows, 256 * 8), 256);
  k_root_hist<IdxT, LabT><<<dim3(blocks, n_slots), 256, C * sizeof(uint32_t), st>>>(v, L.n_in, slot_lo, hist);
  const size_t smask = L.mask[cur] ? (size_t)L.mask_words * sizeof(uint64_t) : 0;
  k_root<IdxT, LabT><<<n_slots, 128, smask, st>>>(v, L.n_in, slot_lo, seed, tree_lo, tv, hist, L.list[cur],
                                                  L.tot[cur], L.cap_list, L.s.ctr, L.mask[cur]);
  current_prof()->launched(CT_K_CHILDREN, 2);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int root(const ct_problem* p, const View& v, const FitLayout& L, uint32_t slot_lo, uint32_t n_slots,
         uint32_t tree_lo, const TreeView& tv, int cur, cudaStream_t st) {
  const uint32_t ib = p->index_bytes, lb = p->label_bytes;
  if (ib == 2 && lb == 1)
    return launch_root<uint16_t, uint8_t>(v, L, slot_lo, n_slots, p->seed, tree_lo, tv, cur, st);
  if (ib == 2 && lb == 2)
    return launch_root<uint16_t, uint16_t>(v, L, slot_lo, n_slots, p->seed, tree_lo, tv, cur, st);
  if (ib == 4 && lb == 1)
    return launch_root<uint32_t, uint8_t>(v, L, slot_lo, n_slots, p->seed, tree_lo, tv, cur, st);
  return launch_root<uint32_t, uint16_t>(v, L, slot_lo, n_slots, p->seed, tree_lo, tv, cur, st);
}

// Grow the warp subtrees of every small node set aside so far.  Their rows
// stay valid in their list buffer: later steps write only other nodes'
// (disjoint) ranges.  Deferring them to one launch lets long subtrees overlap.
int flush_subtrees(const ct_problem* p, const View& v, const FitLayout& L, const TreeView& tv, cudaStream_t st) {
  if (!L.subtree_cut || L.small_bound == 0) return CT_OK;
  CT_TRY(launch_subtrees(v, p->index_bytes, p->label_bytes, L.small, L.cap_small,
                         (uint32_t)std::min<uint64_t>(L.small_bound, L.cap_small), L.subtree_cut > 32, false, L.s, tv,
                         st));
  CT_CUDA_TRY(cudaMemsetAsync(&L.s.ctr->n_small, 0, sizeof(uint32_t), st));
  L.small_bound = 0;
  return CT_OK;
}

// The lists of a step over list[cur][lo..): children go to list[1 - cur].
StepLists step_lists(const FitLayout& L, int cur, uint32_t lo, uint32_t C, uint64_t level_samples) {
  StepLists sl;
  sl.scan_piece = step_piece(level_samples, L.scan_piece, L.mat16);
  sl.nodes = L.list[cur] + lo;
  sl.tot = L.tot[cur] + (size_t)lo * C;
  sl.node_mask = L.mask[cur] ? L.mask[cur] + (size_t)lo * L.mask_words : nullptr;
  sl.next = L.list[1 - cur];
  sl.next_tot = L.tot[1 - cur];
  sl.next_mask = L.mask[1 - cur];
  return sl;
}

// One step over list[cur][0..n) -> children appended to list[1-cur].
int step(const ct_problem* p, const View& v, const FitLayout& L, const TreeView& tv, int cur, uint32_t n,
         uint64_t total, cudaStream_t st) {
  const uint32_t ib = p->index_bytes, lb = p->label_bytes, C = p->n_classes;
  for (uint32_t lo = 0; lo < n; lo += L.chunk) {
    const uint32_t cn = std::min(L.chunk, n - lo);
    const LevelBounds b{cn, total};
    if (L.subtree_cut && L.small_bound + 2ull * cn > L.cap_small) CT_TRY(flush_subtrees(p, v, L, tv, st));
    CT_TRY(launch_reset_step(L.s, cn, step_lists(L, cur, lo, C, total), st));
    // Persistent split and children launches (at most the resident blocks):
    // their grids would otherwise be sized by the capacity bounds, most of
    // whose warps find no item.  The mark fill keeps one warp per piece.
    CT_TRY(launch_split(v, ib, lb, L.s, b, L.scan_piece, true, st));
    CT_TRY(launch_partition(v, ib, lb, L.s, b, tv, false, st));
    CT_TRY(launch_children(v, ib, lb, L.s, b, tv, L.cap_list, L.subtree_cut, L.small, L.cap_small, true, st));
    if (L.subtree_cut) L.small_bound += 2ull * cn;
  }
  return CT_OK;
}

int level_loop(const ct_problem* p, const View& v, const FitLayout& L, const TreeView& tv, int cur,
               uint32_t n, uint64_t total, cudaStream_t st) {
  Counters h;
  while (n > 0) {
    begin_level(L.s.ctr, st);
    CT_CUDA_TRY(cudaGetLastError());
    CT_TRY(step(p, v, L, tv, cur, n, total, st));
    CT_TRY(read_counters(L, &h, st));
    account_level(p, v, h);
    if (L.subtree_cut) L.small_bound = h.n_small;
    n = h.n_next;
    total = h.next_total;
    cur = 1 - cur;
  }
  return CT_OK;
}

// ---------------------------------------------------------------------------
// Graph-driven level loop of the batched form.
//
// The host-driven loop above reads the step counters after every level to
// learn the next level's size: the reference's per-level round trip
// (random_tree.py:428-431).  Here the loop is one CUDA graph: a conditional
// WHILE node whose body is one step (one chunk of a level), launched
// persistently (at most the resident blocks; warps loop over the items).  A
// kernel at the top of the body points the step's lists at the current
// chunk; one at the bottom advances to the next chunk or, at the end of a
// level, swaps the list buffers, adds the level's counts to the totals and
// sets the loop condition to "the next level has nodes" (0 on a device
// error).  The warp-subtree launches follow the loop in the same graph.  The
// host launches the graph and synchronizes once.
struct LoopLists {
  ct_node* list[2];
  uint32_t* tot[2];
  uint64_t* mask[2];
  uint32_t mask_words;
};

// The level the loop starts with is the last step's children (the roots, or
// the host-driven levels' last children): n_next nodes in list ctl->cur,
// which the host sets before launching the graph.
__global__ void k_loop_init(LoopCtl* ctl, Counters* c, uint32_t cap_list, cudaGraphConditionalHandle h) {
  const uint32_t n = c->error ? 0u : min(c->n_next, cap_list);
  ctl->lo = 0;
  ctl->n_level = n;
  ctl->levels = 0;
  ctl->steps = 0;
  ctl->scan_elems = 0;
  ctl->split_total = 0;
  ctl->part_elems = 0;
  ctl->vrows = 0;
  ctl->level_samples = c->next_total;
  reset_level_counters(c);
  c->claim[ITEM_SUBTREE] = 0;
  c->claim[ITEM_SUBTREE_WIDE] = 0;
  cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
}

__global__ void k_loop_step(LoopCtl* ctl, Counters* c, StepLists* step, LoopLists ll, uint32_t chunk, uint32_t C,
                            uint32_t scan_piece, uint32_t mat16) {
  const uint32_t cur = ctl->cur, lo = ctl->lo;
  reset_step_counters(c, min(chunk, ctl->n_level - lo));
  StepLists sl;
  sl.nodes = ll.list[cur] + lo;
  sl.tot = ll.tot[cur] + (size_t)lo * C;
  sl.node_mask = ll.mask[cur] ? ll.mask[cur] + (size_t)lo * ll.mask_words : nullptr;
  sl.next = ll.list[cur ^ 1u];
  sl.next_tot = ll.tot[cur ^ 1u];
  sl.next_mask = ll.mask[cur ^ 1u];
  sl.scan_piece = step_piece(ctl->level_samples, scan_piece, mat16);
  *step = sl;
}

__global__ void k_loop_end(LoopCtl* ctl, Counters* c, uint32_t chunk, uint32_t cap_list,
                           cudaGraphConditionalHandle h) {
  ctl->steps += 1;
  if (c->error) {
    cudaGraphSetConditional(h, 0u);
    return;
  }
  if (ctl->lo + chunk < ctl->n_level) {  // more chunks of this level; the condition stays set
    ctl->lo += chunk;
    return;
  }
  ctl->scan_elems += c->scan_elems;
  ctl->split_total += c->split_total;
  ctl->part_elems += c->part_elems;
  ctl->vrows += c->vrows;
  ctl->levels += 1;
  const uint32_t n = min(c->n_next, cap_list);
  ctl->n_level = n;
  ctl->cur ^= 1u;
  ctl->lo = 0;
  ctl->level_samples = c->next_total;
  reset_level_counters(c);
  cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
}

// The instantiated loop graph of the last batched fit on this thread, reused
// while every kernel argument is the same (same problem, workspace, lists and
// options).
struct LoopGraph {
  std::vector<unsigned char> key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = -1;
  ct_kernel_stats per_step{};  // launches of one body iteration
  ct_kernel_stats once{};      // launches outside the loop
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key.clear();
  }
  ~LoopGraph() { reset(); }
};
thread_local LoopGraph t_loop_graph;

template <typename T>
void key_add(std::vector<unsigned char>& k, const T& v) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), b, b + sizeof(T));
}

ct_kernel_stats stats_diff(const ct_kernel_stats& a, const ct_kernel_stats& b) {
  ct_kernel_stats d{};
  for (int i = 0; i < CT_NUM_KERNEL_GROUPS; ++i) d.launches[i] = a.launches[i] - b.launches[i];
  d.total_launches = a.total_launches - b.total_launches;
  return d;
}

// Capture one batch of launches into graph g (after `dep` when given); the
// stream capture is always ended, whatever the launches return.
template <typename F>
int capture_into(cudaGraph_t g, const cudaGraphNode_t* dep, cudaStream_t st, F launches) {
  CT_CUDA_TRY(cudaStreamBeginCaptureToGraph(st, g, dep, nullptr, dep ? 1 : 0, cudaStreamCaptureModeRelaxed));
  const int rc = launches();
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &out);
  if (rc != CT_OK) return rc;
  CT_CUDA_TRY(e);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

// Stream the loop graph is captured on: capture cannot start on the legacy
// default stream, which callers often pass; the graph runs on the caller's.
cudaStream_t capture_stream() {
  static thread_local struct Holder {
    cudaStream_t st = nullptr;
    ~Holder() {
      if (st) cudaStreamDestroy(st);
    }
  } h;
  if (!h.st) cudaStreamCreateWithFlags(&h.st, cudaStreamNonBlocking);
  return h.st;
}

int build_loop_graph(const ct_problem* p, const View& v, const FitLayout& L, const TreeView& tv, cudaStream_t st,
                     LoopGraph& lg) {
  const uint32_t ib = p->index_bytes, lb = p->label_bytes, C = p->n_classes;
  const LevelBounds b{L.chunk, (uint64_t)L.n_slots * p->n_rows};
  const LoopLists ll{{L.list[0], L.list[1]}, {L.tot[0], L.tot[1]}, {L.mask[0], L.mask[1]}, L.mask_words};
  Prof* pf = current_prof();
  CT_CUDA_TRY(cudaGraphCreate(&lg.graph, 0));
  cudaGraphConditionalHandle h;
  CT_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, lg.graph, 0, cudaGraphCondAssignDefault));
  const ct_kernel_stats s0 = pf->stats;
  CT_TRY(capture_into(lg.graph, nullptr, st, [&]() -> int {
    k_loop_init<<<1, 1, 0, st>>>(L.ctl, L.s.ctr, L.cap_list, h);
    pf->launched(CT_K_CHILDREN);
    return CT_OK;
  }));
  cudaGraphNode_t init = nullptr;
  size_t n_nodes = 1;
  CT_CUDA_TRY(cudaGraphGetNodes(lg.graph, &init, &n_nodes));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t loop = nullptr;
  CT_CUDA_TRY(cudaGraphAddNode(&loop, lg.graph, &init, 1, &cp));
  const ct_kernel_stats s1 = pf->stats;
  CT_TRY(capture_into(cp.conditional.phGraph_out[0], nullptr, st, [&]() -> int {
    k_loop_step<<<1, 1, 0, st>>>(L.ctl, L.s.ctr, L.s.step, ll, L.chunk, C, L.scan_piece, L.mat16);
    pf->launched(CT_K_CHILDREN);
    CT_TRY(launch_split(v, ib, lb, L.s, b, L.scan_piece, true, st));
    CT_TRY(launch_partition(v, ib, lb, L.s, b, tv, true, st));
    CT_TRY(launch_children(v, ib, lb, L.s, b, tv, L.cap_list, L.subtree_cut, L.small, L.cap_small, true, st));
    k_loop_end<<<1, 1, 0, st>>>(L.ctl, L.s.ctr, L.chunk, L.cap_list, h);
    pf->launched(CT_K_CHILDREN);
    return CT_OK;
  }));
  const ct_kernel_stats s2 = pf->stats;
  CT_TRY(capture_into(lg.graph, &loop, st, [&]() -> int {
    return launch_subtrees(v, ib, lb, L.small, L.cap_small, L.cap_small, L.subtree_cut > 32, true, L.s, tv, st);
  }));
  const ct_kernel_stats s3 = pf->stats;
  lg.per_step = stats_diff(s2, s1);
  lg.once = stats_diff(s1, s0);
  const ct_kernel_stats tail = stats_diff(s3, s2);
  for (int i = 0; i < CT_NUM_KERNEL_GROUPS; ++i) lg.once.launches[i] += tail.launches[i];
  lg.once.total_launches += tail.total_launches;
  pf->stats = s0;  // the capture launched nothing; executions are counted after they run
  CT_CUDA_TRY(cudaGraphInstantiate(&lg.exec, lg.graph, 0));
  return CT_OK;
}

// Level loop + warp subtrees of a batched fit as one graph launch, from the
// level of list `cur` on.
int graph_level_loop(const ct_problem* p, const View& v, const FitLayout& L, const TreeView& tv, int cur,
                     cudaStream_t st) {
  std::vector<unsigned char> key;
  int dev = -1;
  CT_CUDA_TRY(cudaGetDevice(&dev));
  key_add(key, dev);
  key_add(key, v);
  key_add(key, L.s);
  key_add(key, tv);
  key_add(key, *p);
  for (int i = 0; i < 2; ++i) {
    key_add(key, L.list[i]);
    key_add(key, L.tot[i]);
    key_add(key, L.mask[i]);
  }
  key_add(key, L.ctl);
  key_add(key, L.small);
  key_add(key, L.cap_small);
  key_add(key, L.cap_list);
  key_add(key, L.chunk);
  key_add(key, L.n_slots);
  key_add(key, L.scan_piece);
  key_add(key, L.mat16);
  key_add(key, L.subtree_cut);
  LoopGraph& lg = t_loop_graph;
  if (!lg.exec || lg.key != key) {
    lg.reset();
    cudaStream_t cs = capture_stream();
    if (!cs) {
      set_last_error("could not create the loop graph's capture stream");
      return CT_ERR_CUDA;
    }
    const int rc = build_loop_graph(p, v, L, tv, cs, lg);
    if (rc != CT_OK) {
      lg.reset();
      return rc;
    }
    lg.key = key;
    lg.device = dev;
  }
  // the loop starts from list `cur` (k_loop_init keeps ctl->cur)
  CT_CUDA_TRY(cudaMemsetAsync(&L.ctl->cur, 0, sizeof(uint32_t), st));
  if (cur) CT_CUDA_TRY(cudaMemsetAsync(&L.ctl->cur, 1, 1, st));
  CT_CUDA_TRY(cudaGraphLaunch(lg.exec, st));
  LoopCtl ctl;
  Counters h;
  CT_CUDA_TRY(cudaMemcpyAsync(&ctl, L.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st));
  CT_TRY(read_counters(L, &h, st));
  Prof* pf = current_prof();
  for (int i = 0; i < CT_NUM_KERNEL_GROUPS; ++i)
    pf->stats.launches[i] += lg.once.launches[i] + (uint64_t)ctl.steps * lg.per_step.launches[i];
  pf->stats.total_launches += lg.once.total_launches + (uint64_t)ctl.steps * lg.per_step.total_launches;
  Counters tot{};
  tot.scan_elems = ctl.scan_elems;
  tot.split_total = ctl.split_total;
  tot.part_elems = ctl.part_elems;
  tot.vrows = ctl.vrows;
  const uint64_t steps = pf->stats.steps;
  account_level(p, v, tot);
  pf->stats.steps = steps + ctl.levels;
  return CT_OK;
}

TreeView tree_view(const ct_tree_buffers* t, uint32_t slot_base) {
  TreeView tv;
  tv.left = t->left;
  tv.right = t->right;
  tv.feature = t->feature;
  tv.threshold = t->threshold;
  tv.value = t->value;
  tv.n_nodes = t->n_nodes;
  tv.capacity = t->capacity;
  tv.slot_base = slot_base;
  tv.enabled = 1;
  return tv;
}

uint32_t default_bfs_threshold(const ct_problem* p) {
  // reference random_forest.py:278-289 ("Titan" coefficients)
  double t = 4746.0 + 4.0 * p->n_classes + 0.0651 * p->n_rows - 75.0 * p->max_features;
  long v = (long)t;
  v = std::min<long>(v, 50000);
  v = std::max<long>(v, 2000);
  return (uint32_t)v;
}

// The fit's view: list entries carry their row's label when it fits
// (fit_label_shift), and two-valued features are marked (feature_flags, run
// at the start of each fit call) for the split scan's boundary search.  The
// packed presort that seeds the lists goes to slot 0 of buffer 1, which no
// step writes before the first partition.
View fit_view(const ct_problem* p, const ct_lists* l, const FitLayout& L) {
  View v = make_view(p, l);
  if (const uint32_t sh = fit_label_shift(p)) {
    v.lab_shift = sh;
    v.row_mask = (1u << sh) - 1u;
  }
  v.fbin = L.fbin;
  return v;
}

// Per-feature preparation of a fit call: the two-valued features; when the
// fit can have virtual features, which ones are (every two-valued feature
// but feature 0, whose lists give the leaf labels) and their rows' value
// bits; and whether a batched fit of more than 64 features keeps
// constant-feature masks.  With few-valued features, lists go constant in
// big nodes and the masks save their partition; with continuous features
// they rarely do, and k_children would only pay for the checks.
// Two-valued features stand for the few-valued ones: masks are kept when at
// least one feature in eight is two-valued.
int prepare_features(const ct_problem* p, FitLayout* L, View* v, cudaStream_t st) {
  CT_TRY(feature_flags(p->x_fm, p->n_rows, p->n_features, L->fbin, L->virt ? L->vval : nullptr, L->ffwork, st));
  if (L->mask[0] && p->n_features > 64) {
    std::vector<uint32_t> fb((p->n_features + 31) / 32);
    CT_CUDA_TRY(cudaMemcpyAsync(fb.data(), L->fbin, fb.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t two = 0;
    for (uint32_t w : fb) two += (uint64_t)__builtin_popcount(w);
    if (two * 8 < p->n_features) L->mask[0] = L->mask[1] = nullptr;
  }
  if (!L->virt) return CT_OK;
  const FitLayout& Lc = *L;
  uint32_t fb[2] = {0, 0};
  CT_CUDA_TRY(cudaMemcpyAsync(fb, Lc.fbin, ((p->n_features + 31) / 32) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t all = p->n_features >= 64 ? ~0ull : (1ull << p->n_features) - 1ull;
  const uint64_t vm = (((uint64_t)fb[1] << 32) | fb[0]) & all & ~1ull;
  if (!vm) return CT_OK;
  v->vmask = vm;
  v->vslot = (uint32_t)__builtin_ctzll(vm);
  // virtual features make no scan pieces: a node scans m (F - virtual) / F lists on average
  const uint64_t mat = (uint64_t)p->n_features - (uint64_t)__builtin_popcountll(vm);
  L->mat16 = (uint32_t)std::max<uint64_t>(1, 16ull * std::min(p->max_features, p->n_features) * mat / p->n_features);
  v->vrow = Lc.vrow;
  v->vval = Lc.vval;
  return virtual_rows(p->x_fm, p->n_rows, vm, Lc.vval, Lc.vrow, st);
}

int seed_source(const ct_problem* p, const ct_lists* l, const View& v, const void** src, cudaStream_t st) {
  *src = p->presort;
  if (v.lab_shift) {
    CT_TRY(pack_presort(p, l->si1, v.lab_shift, v.vmask ? v.vslot : NONE, virtual_skip(v), st));
    *src = l->si1;
  }
  return CT_OK;
}

int fit_batched(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees,
                const FitLayout& L0, const ct_tree_buffers* trees, cudaStream_t st) {
  FitLayout L = L0;
  View v = fit_view(p, l, L);
  TreeView tv = tree_view(trees, 0);
  CT_TRY(prepare_features(p, &L, &v, st));
  CT_CUDA_TRY(cudaMemsetAsync(L.s.ctr, 0, sizeof(Counters), st));
  CT_CUDA_TRY(cudaMemsetAsync(L.boot_ws, 0, 16, st));
  current_prof()->begin(CT_K_BOOTSTRAP);
  const void* src = nullptr;
  CT_TRY(seed_source(p, l, v, &src, st));
  CT_TRY(bootstrap_many(p, l, 0, n_trees, first_tree, src, v.row_mask, virtual_skip(v), L.n_in, L.boot_ws,
                        L.boot_bytes, st));
  current_prof()->end();
  for (uint32_t s = 0; s < n_trees; ++s) account_bootstrap(p, virtual_skip(v));
  CT_TRY(check_boot_error(L, st));
  begin_level(L.s.ctr, st);
  CT_TRY(root(p, v, L, 0, n_trees, first_tree, tv, 0, st));
  Counters h;
  if (!current_prof()->timing && !L.host_loop) {
    // Levels holding more than graph_samples samples run from the host (one
    // round trip each); the rest, and the subtrees, run as the loop graph.
    uint32_t n = 0;
    uint64_t total = 0;
    if (L.graph_samples != UINT64_MAX) {
      CT_TRY(read_counters(L, &h, st));
      n = h.n_next;
      total = h.next_total;
    }
    int cur = 0;
    while (n > 0 && total > L.graph_samples) {
      begin_level(L.s.ctr, st);
      CT_TRY(step(p, v, L, tv, cur, n, total, st));
      CT_TRY(read_counters(L, &h, st));
      account_level(p, v, h);
      if (L.subtree_cut) L.small_bound = h.n_small;
      n = h.n_next;
      total = h.next_total;
      cur = 1 - cur;
    }
    return graph_level_loop(p, v, L, tv, cur, st);
  }
  // host-driven: per-level CUDA-event timing (profiled fits) needs the levels as separate launches
  CT_TRY(read_counters(L, &h, st));
  CT_TRY(level_loop(p, v, L, tv, 0, h.n_next, h.next_total, st));
  if (L.small_bound) {
    CT_TRY(flush_subtrees(p, v, L, tv, st));
    CT_TRY(read_counters(L, &h, st));
  }
  return CT_OK;
}

int fit_plain(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees,
              const ct_fit_options* o, const FitLayout& L0, const ct_tree_buffers* trees,
              cudaStream_t st) {
  FitLayout L = L0;
  View v = fit_view(p, l, L);
  const uint32_t C = p->n_classes;
  const uint32_t thr = o->bfs_threshold ? o->bfs_threshold : default_bfs_threshold(p);
  CT_TRY(prepare_features(p, &L, &v, st));
  struct Pending {
    ct_node nd;
    std::vector<uint32_t> tot;
  };
  CT_CUDA_TRY(cudaMemsetAsync(L.s.ctr, 0, sizeof(Counters), st));
  for (uint32_t t = 0; t < n_trees; ++t) {
    TreeView tv = tree_view(trees, t);
    CT_CUDA_TRY(cudaMemsetAsync(L.boot_ws, 0, 16, st));
    current_prof()->begin(CT_K_BOOTSTRAP);
    const void* src = nullptr;  // packed again per tree: the previous tree's steps wrote buffer 1
    CT_TRY(seed_source(p, l, v, &src, st));
    CT_TRY(bootstrap_many(p, l, 0, 1, first_tree + t, src, v.row_mask, virtual_skip(v), L.n_in, L.boot_ws,
                          L.boot_bytes, st));
    current_prof()->end();
    account_bootstrap(p, virtual_skip(v));
    CT_TRY(check_boot_error(L, st));
    begin_level(L.s.ctr, st);
    CT_TRY(root(p, v, L, 0, 1, first_tree + t, tv, 0, st));
    Counters h;
    CT_TRY(read_counters(L, &h, st));
    if (h.n_next == 0) continue;
    std::vector<Pending> stack, bfs;
    Pending r;
    r.tot.resize(C);
    CT_CUDA_TRY(cudaMemcpyAsync(&r.nd, L.list[0], sizeof(ct_node), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaMemcpyAsync(r.tot.data(), L.tot[0], C * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    stack.push_back(std::move(r));
    while (!stack.empty()) {
      Pending cur = std::move(stack.back());
      stack.pop_back();
      if (cur.nd.n <= thr) {
        bfs.push_back(std::move(cur));
        continue;
      }
      CT_CUDA_TRY(cudaMemcpyAsync(L.list[0], &cur.nd, sizeof(ct_node), cudaMemcpyHostToDevice, st));
      CT_CUDA_TRY(cudaMemcpyAsync(L.tot[0], cur.tot.data(), C * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
      begin_level(L.s.ctr, st);
      CT_TRY(step(p, v, L, tv, 0, 1, cur.nd.n, st));
      CT_TRY(read_counters(L, &h, st));
      account_level(p, v, h);
      if (L.subtree_cut) L.small_bound = h.n_small;
      std::vector<ct_node> kids(h.n_next);
      std::vector<uint32_t> ktot((size_t)h.n_next * C);
      if (h.n_next) {
        CT_CUDA_TRY(cudaMemcpyAsync(kids.data(), L.list[1], h.n_next * sizeof(ct_node),
                                    cudaMemcpyDeviceToHost, st));
        CT_CUDA_TRY(cudaMemcpyAsync(ktot.data(), L.tot[1], ktot.size() * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st));
        CT_CUDA_TRY(cudaStreamSynchronize(st));
      }
      // depth-first, left subtree first: push the right child below the left
      std::vector<uint32_t> order(h.n_next);
      for (uint32_t i = 0; i < h.n_next; ++i) order[i] = i;
      std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return kids[a].start > kids[b].start; });
      for (uint32_t i : order) {
        Pending c;
        c.nd = kids[i];
        c.tot.assign(ktot.begin() + (size_t)i * C, ktot.begin() + (size_t)(i + 1) * C);
        stack.push_back(std::move(c));
      }
    }
    if (!bfs.empty()) {
      if (bfs.size() > L.cap_list) {
        set_last_error("BFS queue exceeds list capacity");
        return CT_ERR_CAPACITY;
      }
      std::vector<ct_node> nodes(bfs.size());
      std::vector<uint32_t> tots(bfs.size() * C);
      uint64_t total = 0;
      for (size_t i = 0; i < bfs.size(); ++i) {
        nodes[i] = bfs[i].nd;
        std::memcpy(&tots[i * C], bfs[i].tot.data(), C * sizeof(uint32_t));
        total += bfs[i].nd.n;
      }
      CT_CUDA_TRY(cudaMemcpyAsync(L.list[0], nodes.data(), nodes.size() * sizeof(ct_node),
                                  cudaMemcpyHostToDevice, st));
      CT_CUDA_TRY(cudaMemcpyAsync(L.tot[0], tots.data(), tots.size() * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice, st));
      CT_TRY(level_loop(p, v, L, tv, 0, (uint32_t)nodes.size(), total, st));
    }
    if (L.small_bound) {  // this tree's subtrees, before the next tree reuses the slot
      CT_TRY(flush_subtrees(p, v, L, tv, st));
      CT_TRY(read_counters(L, &h, st));
    }
  }
  return CT_OK;
}

}  // namespace

// Autotuner candidates.  Every option here grows the same trees, so they are
// chosen by timing.  The batched form is tuned in three stages, each around
// the choice before it: the scan piece length x the warp-subtree cutoff
// with the default partition; the partition shape of big segments (tile,
// ring buffers, CTAs per SM) x the size from which a node partitions with
// its tree's mark bits in shared memory; the size up to which a node
// partitions one warp per (node, 8 features).  The plain form tunes the
// depth-first/breadth-first switch (the quantity the reference fits offline,
// estimate_threshold.py, and predicts with random_forest.py:278-289).
std::vector<ct_fit_options> tune_candidates(const ct_problem* p, uint32_t mode, int stage,
                                            const ct_fit_options& base) {
  std::vector<ct_fit_options> c;
  if (mode == CT_FIT_BATCHED && stage == 0) {
    // the defaults first: a later candidate must beat the current best by 1 %
    std::vector<std::pair<uint32_t, uint32_t>> pairs = {{2048u, 32u}};
    for (uint32_t sp : {1024u, 2048u, 4096u})
      for (uint32_t cut : {0u, 32u, 128u})
        if (!(sp == 2048u && cut == 32u)) pairs.push_back({sp, cut});
    for (const auto& pc : pairs) {
      ct_fit_options o{};
      o.mode = CT_FIT_BATCHED;
      o.scan_piece = pc.first;
      o.subtree_cutoff = pc.second;
      c.push_back(o);
    }
  } else if (mode == CT_FIT_BATCHED && stage == 2) {
    for (uint32_t small : {0u, 512u, 2048u, 8192u}) {
      ct_fit_options o = base;
      o.small_rows = small;
      c.push_back(o);
    }
  } else if (mode == CT_FIT_BATCHED && stage == 1) {
    for (uint32_t shape = 0; shape < CT_PART_SHAPES; ++shape)
      for (uint32_t huge : {0u, 16384u, 0xffffffffu}) {
        ct_fit_options o = base;
        o.part_shape = shape;
        o.huge_rows = huge;
        c.push_back(o);
      }
  } else if (stage == 0) {
    // the reference's regression first (the base a candidate must beat by 1 %)
    std::vector<uint32_t> thr = {default_bfs_threshold(p)};
    for (uint32_t t : {2000u, 8000u, 32000u, std::max(2u, p->n_rows)})
      if (std::find(thr.begin(), thr.end(), t) == thr.end()) thr.push_back(t);
    for (uint32_t t : thr) {
      ct_fit_options o{};
      o.mode = CT_FIT_PLAIN;
      o.bfs_threshold = t;
      o.subtree_cutoff = 32;
      c.push_back(o);
    }
  }
  return c;
}

size_t fit_workspace_bytes(const ct_problem* p, uint32_t n_trees, const ct_fit_options* o);
int fit(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees,
        const ct_fit_options* o, const ct_tree_buffers* trees, void* ws, size_t wsb, cudaStream_t st);

// The second stage changes no capacity, so the first stage's candidates bound the workspace.
size_t autotune_workspace_bytes(const ct_problem* p, uint32_t n_trees, uint32_t mode) {
  size_t most = 0;
  for (const ct_fit_options& o : tune_candidates(p, mode, 0, ct_fit_options{}))
    most = std::max(most, fit_workspace_bytes(p, n_trees, &o));
  return most;
}

int autotune(const ct_problem* p, const ct_lists* l, uint32_t n_trees, uint32_t mode, const ct_tree_buffers* trees,
             void* ws, size_t wsb, ct_fit_options* best, float* best_ms, cudaStream_t st) {
  CT_ARG_CHECK(best && (mode == CT_FIT_PLAIN || mode == CT_FIT_BATCHED), "autotune: bad arguments");
  cudaEvent_t e0, e1;
  CT_CUDA_TRY(cudaEventCreate(&e0));
  CT_CUDA_TRY(cudaEventCreate(&e1));
  float top = 3.0e38f;
  int rc = CT_OK;
  bool any = false;
  for (int stage = 0; stage < 3 && rc == CT_OK; ++stage) {
    if (stage > 0 && !any) break;
    const ct_fit_options base = *best;
    bool first = true;  // a stage's first candidate is its base (or the defaults), timed again
    for (const ct_fit_options& o : tune_candidates(p, mode, stage, base)) {
      if (fit_workspace_bytes(p, n_trees, &o) > wsb) continue;
      float t = 3.0e38f;
      for (int rep = 0; rep < 2 && rc == CT_OK; ++rep) {
        cudaEventRecord(e0, st);
        rc = fit(p, l, 0, n_trees, &o, trees, ws, wsb, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = CT_ERR_CUDA;
        float ms = 0.f;
        if (rc == CT_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) t = std::min(t, ms);
      }
      if (rc != CT_OK) break;
      // timing noise is a few tenths of a percent to 1 %: the base stays
      // unless another candidate beats it by more
      if (first || t < 0.99f * top) {
        top = t;
        *best = o;
        any = true;
      }
      first = false;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != CT_OK) return rc;
  if (!any) {
    set_last_error("autotune: workspace too small for every candidate");
    return CT_ERR_OOM;
  }
  if (best_ms) *best_ms = top;
  return CT_OK;
}

size_t fit_workspace_bytes(const ct_problem* p, uint32_t n_trees, const ct_fit_options* o) {
  FitLayout L;
  layout(p, n_trees, o, nullptr, 0, &L);
  return L.bytes;
}

int fit(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees,
        const ct_fit_options* o, const ct_tree_buffers* trees, void* ws, size_t wsb, cudaStream_t st) {
  CT_TRY(check_problem(p));
  CT_ARG_CHECK(l && l->si0 && l->si1 && l->mark, "lists are NULL");
  CT_ARG_CHECK(trees && trees->left && trees->right && trees->feature && trees->threshold && trees->value &&
                   trees->n_nodes,
               "tree buffers are NULL");
  CT_ARG_CHECK(o && (o->mode == CT_FIT_PLAIN || o->mode == CT_FIT_BATCHED), "bad fit mode");
  CT_ARG_CHECK(o->part_shape < CT_PART_SHAPES, "part_shape out of range");
  CT_ARG_CHECK(o->huge_rows == 0 || o->huge_rows >= CT_HUGE_ROWS_MIN, "huge_rows must be 0 or >= 4096");
  CT_ARG_CHECK(o->small_rows == 0 || (o->small_rows >= 512 && o->small_rows <= 65536),
               "small_rows must be 0 or in [512, 65536]");
  CT_ARG_CHECK(n_trees >= 1, "n_trees must be >= 1");
  CT_ARG_CHECK(trees->capacity >= 2u * p->n_rows, "tree capacity must be >= 2 * n_rows");
  CT_ARG_CHECK(l->stride >= p->n_rows, "list stride must be >= n_rows");
  const uint32_t need_slots = (o->mode == CT_FIT_PLAIN) ? 1u : n_trees;
  CT_ARG_CHECK(l->n_slots >= need_slots, "lists hold too few tree slots");
  FitLayout L;
  if (!layout(p, n_trees, o, reinterpret_cast<char*>(ws), wsb, &L)) {
    set_last_error("fit workspace too small");
    return CT_ERR_OOM;
  }
  Prof* pf = current_prof();
  pf->finish();
  pf->stats = ct_kernel_stats{};
  pf->timing = (o->flags & CT_FIT_PROFILE) != 0;
  pf->st = st;
  const int rc = (o->mode == CT_FIT_PLAIN) ? fit_plain(p, l, first_tree, n_trees, o, L, trees, st)
                                           : fit_batched(p, l, first_tree, n_trees, L, trees, st);
  pf->finish();
  pf->timing = false;
  return rc;
}

// ---------------------------------------------------------------------------
int canonicalize(const uint32_t* left, const uint32_t* right, const uint32_t* feature, const float* threshold,
                 const uint32_t* value, uint32_t n, uint32_t* ol, uint32_t* orr, uint16_t* of, float* ot,
                 uint32_t* ov) {
  CT_ARG_CHECK(n >= 1, "tree has no nodes");
  std::vector<uint32_t> order;
  std::vector<uint32_t> newid(n, NONE);
  order.reserve(n);
  order.push_back(0);
  newid[0] = 0;
  for (size_t h = 0; h < order.size(); ++h) {
    const uint32_t r = order[h];
    if (left[r] != 0 && right[r] != 0) {
      if (left[r] >= n || right[r] >= n || newid[left[r]] != NONE || newid[right[r]] != NONE) {
        set_last_error("raw tree is not a binary tree rooted at node 0");
        return CT_ERR_INTERNAL;
      }
      newid[left[r]] = (uint32_t)order.size();
      order.push_back(left[r]);
      newid[right[r]] = (uint32_t)order.size();
      order.push_back(right[r]);
    }
  }
  if (order.size() != n) {
    set_last_error("raw tree has unreachable nodes");
    return CT_ERR_INTERNAL;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t r = order[i];
    const bool inner = left[r] != 0 && right[r] != 0;
    ol[i] = inner ? newid[left[r]] : 0;
    orr[i] = inner ? newid[right[r]] : 0;
    of[i] = (uint16_t)feature[r];
    ot[i] = threshold[r];
    ov[i] = value[r];
  }
  return CT_OK;
}

// ---------------------------------------------------------------------------
// Read-back of one fit call's trees: the used prefix of every tree's raw
// arrays is gathered into contiguous device arrays (one kernel), copied to
// the host in five transfers, and renumbered breadth-first on host threads.
namespace {

__global__ void k_gather_trees(ct_tree_buffers tb, const uint32_t* __restrict__ off, uint32_t n_trees,
                               uint32_t total, uint32_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n_trees;  // tree t with off[t] <= i < off[t + 1]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (off[mid] <= i) lo = mid; else hi = mid;
    }
    const size_t src = (size_t)lo * tb.capacity + (i - off[lo]);
    out[i] = tb.left[src];
    out[(size_t)total + i] = tb.right[src];
    out[2 * (size_t)total + i] = tb.feature[src];
    out[3 * (size_t)total + i] = __float_as_uint(tb.threshold[src]);
    out[4 * (size_t)total + i] = tb.value[src];
  }
}

// Page-locked staging for the raw read-back, shared by the process and grown
// on demand (portable across devices).  Page-locked allocation synchronizes
// the device and takes tens of ms for a 100-tree forest, so a server reserves
// its largest size up front, and a growth takes half again the old size
// (16 MiB steps): forests a little larger than the last do not reallocate.
struct Staging {
  std::mutex mu;
  void* p = nullptr;
  size_t bytes = 0;
  int grow(size_t need) {  // caller holds mu
    if (bytes >= need) return CT_OK;
    constexpr size_t STEP = size_t(16) << 20;
    const size_t want = (std::max(need, bytes + bytes / 2) + STEP - 1) / STEP * STEP;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    CT_CUDA_TRY(cudaHostAlloc(&p, want, cudaHostAllocPortable));
    bytes = want;
    return CT_OK;
  }
};
Staging g_staging;

}  // namespace

int fetch_trees_reserve(uint64_t total_nodes) {
  std::lock_guard<std::mutex> lk(g_staging.mu);
  return g_staging.grow(5 * total_nodes * sizeof(uint32_t));
}

size_t fetch_trees_scratch(uint64_t total_nodes, uint32_t n_trees) {
  return 5 * total_nodes * sizeof(uint32_t) + ((size_t)n_trees + 1) * sizeof(uint32_t) + 256;
}

int fetch_trees(const ct_tree_buffers* tb, uint32_t n_trees, const uint32_t* counts, void* scratch,
                size_t scratch_bytes, uint32_t* ol, uint32_t* orr, uint16_t* of, float* ot, uint32_t* ov,
                cudaStream_t st) {
  CT_ARG_CHECK(tb && counts && scratch && ol && orr && of && ot && ov, "fetch trees: NULL argument");
  std::vector<uint32_t> off(n_trees + 1, 0);
  for (uint32_t t = 0; t < n_trees; ++t) {
    CT_ARG_CHECK(counts[t] >= 1 && counts[t] <= tb->capacity, "fetch trees: node count out of range");
    CT_ARG_CHECK((uint64_t)off[t] + counts[t] < (1ull << 32), "fetch trees: too many nodes for one call");
    off[t + 1] = off[t] + counts[t];
  }
  const uint32_t total = off[n_trees];
  if (n_trees == 0) return CT_OK;
  CT_ARG_CHECK(scratch_bytes >= fetch_trees_scratch(total, n_trees), "fetch trees: scratch too small");
  uint32_t* d_cols = reinterpret_cast<uint32_t*>(scratch);
  uint32_t* d_off = d_cols + 5 * (size_t)total;
  CT_CUDA_TRY(cudaMemcpyAsync(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st));
  k_gather_trees<<<std::min<uint32_t>(ceil_div(total, 256), 148 * 16), 256, 0, st>>>(*tb, d_off, n_trees, total,
                                                                                    d_cols);
  CT_CUDA_TRY(cudaGetLastError());
  std::lock_guard<std::mutex> lk(g_staging.mu);
  CT_TRY(g_staging.grow((size_t)5 * total * sizeof(uint32_t)));
  CT_CUDA_TRY(cudaMemcpyAsync(g_staging.p, d_cols, (size_t)5 * total * 4, cudaMemcpyDeviceToHost, st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  const uint32_t* hl = static_cast<const uint32_t*>(g_staging.p);
  const uint32_t* hr = hl + total;
  const uint32_t* hf = hr + total;
  const float* ht = reinterpret_cast<const float*>(hf + total);
  const uint32_t* hv = hf + 2 * (size_t)total;
  const uint32_t workers = std::max(1u, std::min({n_trees, 16u, std::thread::hardware_concurrency()}));
  std::vector<int> status(workers, CT_OK);
  std::vector<std::string> errors(workers);
  auto run = [&](uint32_t w) {
    for (uint32_t t = w; t < n_trees; t += workers) {
      const uint32_t o = off[t];
      const int rc = canonicalize(hl + o, hr + o, hf + o, ht + o, hv + o, counts[t], ol + o, orr + o, of + o,
                                  ot + o, ov + o);
      if (rc != CT_OK) {
        status[w] = rc;
        errors[w] = "tree " + std::to_string(t) + ": " + last_error_text();
        return;
      }
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t w = 1; w < workers; ++w) pool.emplace_back(run, w);
  run(0);
  for (auto& th : pool) th.join();
  for (uint32_t w = 0; w < workers; ++w)
    if (status[w] != CT_OK) {
      set_last_error(errors[w]);
      return status[w];
    }
  return CT_OK;
}

// ---------------------------------------------------------------------------
// Forest queue: the batched fit of several independent jobs (each its own
// samples, labels, presort, index lists, F, C, m and seed) through shared
// level steps.  Each job is prepared on its own (feature flags, packed
// presort, bootstrap, roots); from then on one node list holds every job's
// nodes and every level kernel serves all of them, each work item reading
// its job's view (View::jobs).  The tree slots are numbered across the jobs
// in order; a job's trees are the ones its solo fit grows (the same seed,
// tree keys and canonical rule).  The reference runs such a queue as one
// process per job over its GPU (hybridforest/builder.py:79-141).
namespace {

struct QueueShape {
  uint32_t slots = 0;      // trees of all jobs
  uint64_t samples = 0;    // sum over trees of their job's rows
  uint32_t n_max = 0, f_max = 0, c_max = 0, m_max = 0;
  uint32_t fbin_words = 0; // sum over jobs of their flag words
  size_t ff_bytes = 0, boot_bytes = 0;
};

QueueShape queue_shape(const ct_fit_job* jobs, uint32_t n_jobs) {
  QueueShape q;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const ct_problem& p = jobs[j].problem;
    q.slots += jobs[j].n_trees;
    q.samples += (uint64_t)jobs[j].n_trees * p.n_rows;
    q.n_max = std::max(q.n_max, p.n_rows);
    q.f_max = std::max(q.f_max, p.n_features);
    q.c_max = std::max(q.c_max, p.n_classes);
    q.m_max = std::max(q.m_max, p.max_features);
    q.fbin_words += (p.n_features + 31) / 32;
    q.ff_bytes = std::max(q.ff_bytes, feature_flags_work_bytes(p.n_features));
    q.boot_bytes = std::max(q.boot_bytes, bootstrap_scratch_bytes(p.n_rows, p.n_features, jobs[j].n_trees));
  }
  return q;
}

// The batch's problem: the first job's widths, the largest F, C and m of any
// job (the scratch strides), and the largest row count.
ct_problem batch_problem(const ct_fit_job* jobs, const QueueShape& q) {
  ct_problem pb = jobs[0].problem;
  pb.n_rows = q.n_max;
  pb.n_features = q.f_max;
  pb.n_classes = q.c_max;
  pb.max_features = q.m_max;
  return pb;
}

bool layout_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o, char* base, size_t size,
                  FitLayout* L, View** views_dev, uint32_t** slot_job_dev) {
  const QueueShape q = queue_shape(jobs, n_jobs);
  const ct_problem pb = batch_problem(jobs, q);
  View v = make_view(&pb, nullptr);
  L->n_slots = q.slots;
  L->cap_list = (uint32_t)std::min<uint64_t>(q.samples / 2 + q.slots + 2, 0xffffffffull);
  L->chunk = std::min<uint32_t>(L->cap_list, o->step_nodes ? o->step_nodes : CHUNK_NODES_MAX);
  L->scan_piece = o->scan_piece ? o->scan_piece : DEFAULT_SCAN_PIECE;
  L->subtree_cut = q.n_max < (1u << 27) ? std::min<uint32_t>(o->subtree_cutoff, 128u) : 0u;
  L->cap_small = L->subtree_cut ? 2 * L->chunk : 0u;
  L->host_loop = (o->flags & CT_FIT_HOST_LOOP) != 0;
  L->graph_samples = o->graph_samples == 0xffffffffu ? UINT64_MAX
                     : o->graph_samples               ? o->graph_samples
                                                      : DEFAULT_GRAPH_SAMPLES;
  Arena a{base, size, 0};
  L->small = L->cap_small ? a.take<ct_node>(L->cap_small) : nullptr;
  L->small_bound = 0;
  L->n_in = a.take<uint32_t>(q.slots);
  L->fbin = a.take<uint32_t>(q.fbin_words);
  L->ffwork = a.take<char>(q.ff_bytes);
  L->virt = false;
  L->vrow = nullptr;
  L->vval = nullptr;
  // constant-feature masks while every job has at most 64 features
  const bool masks = q.f_max <= 64;
  L->mask_words = mask_words(q.f_max);
  for (int i = 0; i < 2; ++i) {
    L->list[i] = a.take<ct_node>(L->cap_list);
    L->tot[i] = a.take<uint32_t>((size_t)L->cap_list * q.c_max);
    L->mask[i] = masks ? a.take<uint64_t>((size_t)L->cap_list * L->mask_words) : nullptr;
  }
  L->boot_bytes = q.boot_bytes;
  L->boot_ws = a.take<char>(L->boot_bytes);
  L->mat16 = 16 * q.m_max;
  LevelCaps caps = level_caps(v, step_piece(0, L->scan_piece, 1), LevelBounds{L->chunk, q.samples});
  carve_level_scratch(a, v, caps, &L->s, false);
  // jobs of different row counts have mark bits of different sizes: no shared-memory staging
  L->s.huge_segs = nullptr;
  L->s.cap_huge = 0;
  L->s.huge_rows = 0xffffffffu;
  L->s.part_shape = o->part_shape;
  L->s.small_rows = o->small_rows ? o->small_rows : default_small_rows(jobs[0].problem.index_bytes);
  L->ctl = a.take<LoopCtl>(1);
  *views_dev = a.take<View>(n_jobs);
  *slot_job_dev = a.take<uint32_t>(q.slots);
  L->bytes = a.used + 256;
  return base != nullptr && a.ok();
}

}  // namespace

size_t fit_queue_workspace_bytes(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o) {
  FitLayout L;
  View* vd = nullptr;
  uint32_t* sj = nullptr;
  layout_queue(jobs, n_jobs, o, nullptr, 0, &L, &vd, &sj);
  return L.bytes;
}

int check_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o, const ct_tree_buffers* trees) {
  CT_ARG_CHECK(jobs && n_jobs >= 1, "no jobs");
  CT_ARG_CHECK(o && o->mode == CT_FIT_BATCHED, "a forest queue takes the batched form");
  CT_ARG_CHECK(o->part_shape < CT_PART_SHAPES, "part_shape out of range");
  CT_ARG_CHECK(o->small_rows == 0 || (o->small_rows >= 512 && o->small_rows <= 65536),
               "small_rows must be 0 or in [512, 65536]");
  CT_ARG_CHECK(trees && trees->left && trees->right && trees->feature && trees->threshold && trees->value &&
                   trees->n_nodes,
               "tree buffers are NULL");
  uint64_t slots = 0;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const ct_fit_job& jb = jobs[j];
    CT_TRY(check_problem(&jb.problem));
    CT_ARG_CHECK(jb.problem.index_bytes == jobs[0].problem.index_bytes &&
                     jb.problem.label_bytes == jobs[0].problem.label_bytes,
                 "the jobs of one queue fit share index_bytes and label_bytes");
    CT_ARG_CHECK(jb.n_trees >= 1, "a job has no trees");
    CT_ARG_CHECK(jb.lists.si0 && jb.lists.si1 && jb.lists.mark, "a job's lists are NULL");
    CT_ARG_CHECK(jb.lists.stride >= jb.problem.n_rows, "a job's list stride is below its n_rows");
    CT_ARG_CHECK(jb.lists.n_slots >= jb.n_trees, "a job's lists hold too few tree slots");
    CT_ARG_CHECK(trees->capacity >= 2u * jb.problem.n_rows, "tree capacity must be >= 2 * every job's n_rows");
    slots += jb.n_trees;
  }
  CT_ARG_CHECK(slots < (1ull << 31), "too many trees in one queue fit");
  return CT_OK;
}

int fit_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o, const ct_tree_buffers* trees,
              void* ws, size_t wsb, cudaStream_t st) {
  CT_TRY(check_queue(jobs, n_jobs, o, trees));
  FitLayout L;
  View* views_dev = nullptr;
  uint32_t* slot_job_dev = nullptr;
  if (!layout_queue(jobs, n_jobs, o, reinterpret_cast<char*>(ws), wsb, &L, &views_dev, &slot_job_dev)) {
    set_last_error("queue fit workspace too small");
    return CT_ERR_OOM;
  }
  const QueueShape q = queue_shape(jobs, n_jobs);
  const ct_problem pb = batch_problem(jobs, q);
  Prof* pf = current_prof();
  pf->finish();
  pf->stats = ct_kernel_stats{};
  pf->timing = (o->flags & CT_FIT_PROFILE) != 0;
  pf->st = st;
  auto run = [&]() -> int {
    // the jobs' views, with the batch's strides
    std::vector<View> views(n_jobs);
    std::vector<uint32_t> slot_job(q.slots);
    std::vector<uint32_t> first_slot(n_jobs);
    uint32_t slot = 0, fw = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
      const ct_fit_job& jb = jobs[j];
      View vj = fit_view(&jb.problem, &jb.lists, L);
      vj.fbin = L.fbin + fw;
      vj.n_classes = q.c_max;
      vj.slot_base = slot;
      vj.sel_stride = q.m_max;
      vj.mask_stride = L.mask_words;
      views[j] = vj;
      first_slot[j] = slot;
      for (uint32_t t = 0; t < jb.n_trees; ++t) slot_job[slot + t] = j;
      CT_TRY(feature_flags(jb.problem.x_fm, jb.problem.n_rows, jb.problem.n_features, L.fbin + fw, nullptr,
                           L.ffwork, st));
      slot += jb.n_trees;
      fw += (jb.problem.n_features + 31) / 32;
    }
    CT_CUDA_TRY(cudaMemcpyAsync(views_dev, views.data(), n_jobs * sizeof(View), cudaMemcpyHostToDevice, st));
    CT_CUDA_TRY(cudaMemcpyAsync(slot_job_dev, slot_job.data(), q.slots * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                st));
    // the batch view carries the strides; lists and marks are read through
    // the jobs' views (its own point at the first job's, never dereferenced)
    View vb = make_view(&pb, &jobs[0].lists);
    vb.jobs = views_dev;
    vb.slot_job = slot_job_dev;
    vb.sel_stride = q.m_max;
    vb.mask_stride = L.mask_words;
    vb.bit_words = 0;  // per job (the shared-memory staging of marks is off)
    vb.lab_shift = views[0].lab_shift;
    vb.row_mask = views[0].row_mask;
    TreeView tv = tree_view(trees, 0);
    CT_CUDA_TRY(cudaMemsetAsync(L.s.ctr, 0, sizeof(Counters), st));
    CT_CUDA_TRY(cudaMemsetAsync(L.boot_ws, 0, 16, st));
    current_prof()->begin(CT_K_BOOTSTRAP);
    for (uint32_t j = 0; j < n_jobs; ++j) {
      const ct_fit_job& jb = jobs[j];
      const void* src = nullptr;
      CT_TRY(seed_source(&jb.problem, &jb.lists, views[j], &src, st));
      CT_TRY(bootstrap_many(&jb.problem, &jb.lists, 0, jb.n_trees, jb.first_tree, src, views[j].row_mask,
                            virtual_skip(views[j]), L.n_in + first_slot[j], L.boot_ws, L.boot_bytes, st));
      for (uint32_t t = 0; t < jb.n_trees; ++t) account_bootstrap(&jb.problem, virtual_skip(views[j]));
    }
    current_prof()->end();
    CT_TRY(check_boot_error(L, st));
    begin_level(L.s.ctr, st);
    for (uint32_t j = 0; j < n_jobs; ++j)
      CT_TRY(root(&jobs[j].problem, views[j], L, first_slot[j], jobs[j].n_trees, jobs[j].first_tree, tv, 0, st));
    Counters h;
    if (!current_prof()->timing && !L.host_loop) {
      uint32_t n = 0;
      uint64_t total = 0;
      if (L.graph_samples != UINT64_MAX) {
        CT_TRY(read_counters(L, &h, st));
        n = h.n_next;
        total = h.next_total;
      }
      int cur = 0;
      while (n > 0 && total > L.graph_samples) {
        begin_level(L.s.ctr, st);
        CT_TRY(step(&pb, vb, L, tv, cur, n, total, st));
        CT_TRY(read_counters(L, &h, st));
        account_level(&pb, vb, h);
        if (L.subtree_cut) L.small_bound = h.n_small;
        n = h.n_next;
        total = h.next_total;
        cur = 1 - cur;
      }
      return graph_level_loop(&pb, vb, L, tv, cur, st);
    }
    CT_TRY(read_counters(L, &h, st));
    CT_TRY(level_loop(&pb, vb, L, tv, 0, h.n_next, h.next_total, st));
    if (L.small_bound) {
      CT_TRY(flush_subtrees(&pb, vb, L, tv, st));
      CT_TRY(read_counters(L, &h, st));
    }
    return CT_OK;
  };
  const int rc = run();
  pf->finish();
  pf->timing = false;
  return rc;
}

}  // namespace ct
