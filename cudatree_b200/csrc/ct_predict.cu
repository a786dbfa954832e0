// Forest prediction: tree traversal + device-side majority vote.
//
// Reference: predict.cu:12-69 walks one tree per launch with one active lane
// per warp, and random_forest.py:339-362 stacks per-tree labels on the host
// and votes row by row in Python.  Here one launch walks every tree of the
// forest:
//   * blocks cover (row tile, tree group); the trees are cut into groups whose
//     nodes fit comfortably in L2, and blocks are numbered group-major, so the
//     blocks in flight walk one group and its nodes come from DRAM about once
//     per launch instead of once per walk;
//   * walks inside a block are numbered row-fastest: with 32 rows per tile a
//     lane keeps one row and a warp's lanes walk the same tree (shared loads
//     of its top levels); each thread keeps PRED_ILP walks in flight;
//   * the walk is bound by the L1 data path (bytes returned per node visit),
//     so a node is one vector load: 16 bytes in the packed form, 8 bytes in
//     the compact form, which is used whenever a forest's trees fit it;
//   * votes go to a shared-memory histogram; with several groups the
//     histograms are added into a global [rows][classes] table and a second
//     kernel takes the majority, lowest class on ties
//     (np.argmax(np.bincount(...)), random_forest.py:358).
#include <cstring>
#include <mutex>
#include <set>

#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr int PRED_THREADS = 256;
constexpr int PRED_ILP = 8;
constexpr uint32_t X_SMEM_BYTES = 32 * 1024;     // rows of x staged per block when they fit
constexpr uint32_t HIST_SMEM_BYTES = 64 * 1024;  // vote histogram [rows][classes]
constexpr size_t GROUP_L2_BYTES = 32ull << 20;   // node bytes of one tree group

__host__ __device__ __forceinline__ bool predict_rows_staged(uint32_t rpb, uint32_t n_features) {
  return (size_t)rpb * n_features * sizeof(float) <= X_SMEM_BYTES;
}

// Packed form: 16 bytes {threshold, feature, left, value}; left 0 = leaf.
struct PackedForm {
  using Raw = uint4;
  static constexpr size_t BYTES = 16;
  __device__ static Raw load(const void* nodes, uint32_t pos) {
    return __ldg(reinterpret_cast<const uint4*>(nodes) + pos);
  }
  __device__ static bool inner(const Raw& n) { return n.z != 0; }
  __device__ static uint32_t left(const Raw& n, uint32_t) { return n.z; }
  __device__ static uint32_t feature(const Raw& n, uint32_t) { return n.y; }
  __device__ static float threshold(const Raw& n) { return __uint_as_float(n.x); }
  __device__ static uint32_t value(const Raw& n) { return n.w; }
};

// Compact form: 8 bytes; inner {threshold, left << fbits | feature}, leaf
// {class id, 0}.  left >= 1 for inner nodes, so the second word is nonzero.
struct CompactForm {
  using Raw = uint2;
  static constexpr size_t BYTES = 8;
  __device__ static Raw load(const void* nodes, uint32_t pos) {
    return __ldg(reinterpret_cast<const uint2*>(nodes) + pos);
  }
  __device__ static bool inner(const Raw& n) { return n.y != 0; }
  __device__ static uint32_t left(const Raw& n, uint32_t fbits) { return n.y >> fbits; }
  __device__ static uint32_t feature(const Raw& n, uint32_t fbits) { return n.y & ((1u << fbits) - 1u); }
  __device__ static float threshold(const Raw& n) { return __uint_as_float(n.x); }
  __device__ static uint32_t value(const Raw& n) { return n.x; }
};

// Walk every (row, tree) pair of a tile for trees [t_lo, t_lo + n_t) and add
// the leaf votes to hist[row][class].  Feature f of tile row r is
// x[r * row_stride + f * feat_stride]: the staged shared-memory tile is
// feature-major (row_stride 1, feat_stride rpb), so the lanes of a warp, one
// row each, read distinct banks; unstaged rows are read from global memory.
// Walks are numbered w = t * rpb + row (row-fastest); rpb is a power of two
// dividing blockDim.x, so a thread's row is fixed (threadIdx.x % rpb) and its
// tree index advances by blockDim.x / rpb per walk.  Each thread keeps
// PRED_ILP walks in flight; their node loads are issued together, then each
// walk steps or, at a leaf, votes and starts the thread's next tree.
template <typename Form>
__device__ __forceinline__ void walk_tile(const void* __restrict__ nodes, const uint32_t* __restrict__ tree_off,
                                          uint32_t t_lo, uint32_t n_t, uint32_t fbits, const float* x,
                                          uint32_t row_stride, uint32_t feat_stride, uint32_t rows, uint32_t rpb,
                                          uint32_t n_classes, uint32_t* hist) {
  const uint32_t r = threadIdx.x & (rpb - 1);
  if (r >= rows) return;
  const uint32_t t_step = blockDim.x / rpb;
  const float* xr = x + (size_t)r * row_stride;
  uint32_t* hr = hist + r * n_classes;
  uint32_t t_next = threadIdx.x / rpb;
  uint32_t base[PRED_ILP], pos[PRED_ILP];  // pos: absolute node index, NONE when the slot is idle
#pragma unroll
  for (int k = 0; k < PRED_ILP; ++k) {
    pos[k] = NONE;
    base[k] = 0;
    if (t_next < n_t) {
      base[k] = __ldg(tree_off + t_lo + t_next);
      pos[k] = base[k];
      t_next += t_step;
    }
  }
  bool any = pos[0] != NONE;
  while (any) {
    typename Form::Raw nd[PRED_ILP];
#pragma unroll
    for (int k = 0; k < PRED_ILP; ++k)
      if (pos[k] != NONE) nd[k] = Form::load(nodes, pos[k]);
    any = false;
#pragma unroll
    for (int k = 0; k < PRED_ILP; ++k) {
      if (pos[k] == NONE) continue;
      any = true;
      if (Form::inner(nd[k])) {
        const float v = xr[Form::feature(nd[k], fbits) * feat_stride];
        pos[k] = base[k] + Form::left(nd[k], fbits) + (v < Form::threshold(nd[k]) ? 0u : 1u);
      } else {
        atomicAdd(hr + Form::value(nd[k]), 1u);
        pos[k] = NONE;
        if (t_next < n_t) {
          base[k] = __ldg(tree_off + t_lo + t_next);
          pos[k] = base[k];
          t_next += t_step;
        }
      }
    }
  }
}

// Majority of a row's votes, lowest class on ties; warp-collective.
__device__ __forceinline__ uint32_t warp_argmax(const uint32_t* votes, uint32_t n_classes, uint32_t* votes_out) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t best = 0, bc = NONE;
  for (uint32_t c = lane; c < n_classes; c += 32) {
    const uint32_t v = votes[c];
    if (votes_out) votes_out[c] = v;
    if (bc == NONE || v > best) {
      best = v;
      bc = c;
    }
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const uint32_t ob = __shfl_xor_sync(FULL, best, s);
    const uint32_t oc = __shfl_xor_sync(FULL, bc, s);
    if (oc != NONE && (bc == NONE || ob > best || (ob == best && oc < bc))) {
      best = ob;
      bc = oc;
    }
  }
  return bc;
}

// Stage a tile's rows feature-major: xs[f * rpb + r] = x[r][f].  The reads
// are coalesced (x may be mapped host memory, read once over the link); the
// shared-memory stores conflict, which costs far less than the walk's reads.
__device__ __forceinline__ void stage_rows(const float* x, uint32_t rows, uint32_t rpb, uint32_t n_features,
                                           float* xs) {
  for (uint32_t i = threadIdx.x; i < rows * n_features; i += blockDim.x) {
    const uint32_t r = i / n_features, f = i - r * n_features;
    xs[f * rpb + r] = x[i];
  }
}

// One tile of one tree group: walk, then either vote (single group) or add
// the histogram into the global vote table.
template <typename Form>
__device__ __forceinline__ void tile_work(const void* nodes, const uint32_t* tree_off, uint32_t fbits, uint32_t t_lo,
                                          uint32_t n_t, bool single_group, const float* x, uint32_t n_rows,
                                          uint32_t n_features, uint32_t n_classes, uint32_t rpb, uint32_t row0,
                                          uint32_t* votes, uint32_t* pred, uint32_t* smem) {
  uint32_t* hist = smem;
  float* xs = reinterpret_cast<float*>(smem + rpb * n_classes);
  const uint32_t rows = min(rpb, n_rows - row0);
  for (uint32_t i = threadIdx.x; i < rpb * n_classes; i += blockDim.x) hist[i] = 0;
  const bool fits = predict_rows_staged(rpb, n_features);
  if (fits) stage_rows(x + (size_t)row0 * n_features, rows, rpb, n_features, xs);
  __syncthreads();
  if (fits)
    walk_tile<Form>(nodes, tree_off, t_lo, n_t, fbits, xs, 1, rpb, rows, rpb, n_classes, hist);
  else
    walk_tile<Form>(nodes, tree_off, t_lo, n_t, fbits, x + (size_t)row0 * n_features, n_features, 1, rows, rpb,
                    n_classes, hist);
  __syncthreads();
  if (single_group) {
    const uint32_t warp = threadIdx.x >> 5;
    for (uint32_t rr = warp; rr < rows; rr += blockDim.x >> 5) {
      const uint32_t c = warp_argmax(hist + rr * n_classes, n_classes,
                                     votes ? votes + (size_t)(row0 + rr) * n_classes : nullptr);
      if ((threadIdx.x & 31) == 0 && pred) pred[row0 + rr] = c;
    }
  } else {
    for (uint32_t i = threadIdx.x; i < rows * n_classes; i += blockDim.x)
      if (hist[i]) atomicAdd(votes + (size_t)row0 * n_classes + i, hist[i]);
  }
}

template <typename Form>
__global__ void __launch_bounds__(PRED_THREADS, 4)
k_predict(const void* __restrict__ nodes, const uint32_t* __restrict__ tree_off, uint32_t n_trees, uint32_t fbits,
          uint32_t group, uint32_t tiles, const float* __restrict__ x, uint32_t n_rows, uint32_t n_features,
          uint32_t n_classes, uint32_t rpb, uint32_t* __restrict__ votes, uint32_t* __restrict__ pred) {
  extern __shared__ uint32_t smem[];
  const uint32_t g = blockIdx.x / tiles, tile = blockIdx.x - g * tiles;  // group-major
  const uint32_t t_lo = g * group;
  tile_work<Form>(nodes, tree_off, fbits, t_lo, min(group, n_trees - t_lo), group >= n_trees, x, n_rows, n_features,
                  n_classes, rpb, tile * rpb, votes, pred, smem);
}

__global__ void k_vote_rows(const uint32_t* __restrict__ votes, uint32_t n_rows, uint32_t n_classes,
                            uint32_t* __restrict__ pred) {
  const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n_rows) return;
  const uint32_t c = warp_argmax(votes + (size_t)row * n_classes, n_classes, nullptr);
  if ((threadIdx.x & 31) == 0 && pred) pred[row] = c;
}

// A packed node whose child or feature does not fit the compact fields
// becomes an inner node with child 0, which the forest check rejects.
__global__ void k_compact(const ct_packed_node* __restrict__ in, uint32_t n, uint32_t fbits,
                          uint2* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4 p = __ldg(reinterpret_cast<const uint4*>(in) + i);
    const bool fits = (p.z >> (32 - fbits)) == 0u && (p.y >> fbits) == 0u;
    out[i] = p.z ? make_uint2(p.x, fits ? (p.z << fbits) | p.y : 1u) : make_uint2(p.w, 0u);
  }
}

// Forest check before a walk (bits of *err): 1 tree offsets not strictly
// increasing inside [0, n_nodes); 2 an inner node whose left child is not
// after it or whose right child (left + 1) is past its tree; 4 a feature
// index >= n_features; 8 a leaf class >= n_classes.  A forest that passes
// walks every tree in at most its node count of steps (the local index
// strictly increases) and reads only its own nodes, x columns and vote bins.
template <typename Form>
__global__ void k_check_forest(const void* __restrict__ nodes, uint32_t n_nodes, const uint32_t* __restrict__ off,
                               uint32_t n_trees, uint32_t fbits, uint32_t n_features, uint32_t n_classes,
                               uint32_t* err) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  uint32_t bad = 0;
  for (uint32_t t = tid; t < n_trees; t += stride) {
    const uint32_t b = __ldg(off + t), e = t + 1 < n_trees ? __ldg(off + t + 1) : n_nodes;
    if (!(b < e && e <= n_nodes)) bad |= 1u;
  }
  const uint32_t first = __ldg(off);
  for (uint32_t i = tid; i < n_nodes; i += stride) {
    if (i < first) continue;  // before the first tree: never visited
    uint32_t lo = 0, hi = n_trees;  // the tree t with off[t] <= i < off[t + 1]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (__ldg(off + mid) <= i) lo = mid; else hi = mid;
    }
    const uint32_t b = __ldg(off + lo), e = lo + 1 < n_trees ? __ldg(off + lo + 1) : n_nodes;
    if (i < b || i >= e) {  // only when the offsets are out of order (bit 1 is set then)
      bad |= 1u;
      continue;
    }
    const typename Form::Raw nd = Form::load(nodes, i);
    if (Form::inner(nd)) {
      const uint32_t l = Form::left(nd, fbits);
      if (l <= i - b || (uint64_t)l + 1 >= (uint64_t)(e - b)) bad |= 2u;
      if (Form::feature(nd, fbits) >= n_features) bad |= 4u;
    } else if (Form::value(nd) >= n_classes) {
      bad |= 8u;
    }
  }
  if (bad) atomicOr(err, bad);
}

const char* forest_error_text(uint32_t bad) {
  if (bad & 1u) return "tree offsets are not strictly increasing inside the node array";
  if (bad & 2u) return "an inner node's children are not after it inside its tree";
  if (bad & 4u) return "a node's feature index is out of range";
  return "a leaf's class id is out of range";
}

// Checks the forest on the device before a walk.  The check's error word is
// the first word of pred, the caller's output (n_rows >= 1), so nothing is
// allocated; the walk overwrites it.
template <typename Form>
int check_forest_device(const void* nodes, uint32_t n_nodes, const uint32_t* off, uint32_t n_trees, uint32_t fbits,
                        uint32_t n_features, uint32_t n_classes, uint32_t* pred, cudaStream_t st) {
  CT_CUDA_TRY(cudaMemsetAsync(pred, 0, sizeof(uint32_t), st));
  const uint32_t work = std::max(n_nodes, n_trees);
  k_check_forest<Form><<<std::min<uint32_t>(ceil_div(work, 256), 148 * 8), 256, 0, st>>>(
      nodes, n_nodes, off, n_trees, fbits, n_features, n_classes, pred);
  CT_CUDA_TRY(cudaGetLastError());
  uint32_t bad = 0;
  CT_CUDA_TRY(cudaMemcpyAsync(&bad, pred, sizeof(bad), cudaMemcpyDeviceToHost, st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  if (bad) {
    set_last_error(std::string("predict: malformed forest: ") + forest_error_text(bad));
    return CT_ERR_ARG;
  }
  return CT_OK;
}

// Raise a kernel's dynamic shared-memory limit once per device.
template <typename K>
int allow_smem(K kernel, int bytes) {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  CT_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(dev)) return CT_OK;
  CT_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.insert(dev);
  return CT_OK;
}

}  // namespace

// Rows per tile: 32, halved until the [rows][classes] histogram and the
// staged [features][rows] tile fit their shared-memory budgets.
uint32_t predict_rows_per_block(uint32_t n_classes, uint32_t n_features) {
  uint32_t r = 32;
  while (r > 1 && ((size_t)r * n_classes * sizeof(uint32_t) > HIST_SMEM_BYTES ||
                   (size_t)r * n_features * sizeof(float) > X_SMEM_BYTES))
    r >>= 1;
  return r;
}

size_t predict_tile_smem(uint32_t rpb, uint32_t n_classes, uint32_t n_features) {
  return (size_t)rpb * n_classes * sizeof(uint32_t) +
         (predict_rows_staged(rpb, n_features) ? (size_t)rpb * n_features * sizeof(float) : 0);
}

uint32_t predict_group_size(uint32_t n_trees, uint64_t n_nodes, size_t node_bytes) {
  const uint64_t per_tree = (n_nodes * node_bytes + n_trees - 1) / n_trees;
  uint64_t g = per_tree ? GROUP_L2_BYTES / per_tree : n_trees;
  if (g < 1) g = 1;
  return (uint32_t)std::min<uint64_t>(g, n_trees);
}

uint32_t compact_feature_bits(uint32_t n_features) {
  uint32_t b = 1;
  while (b < 31 && (1u << b) < n_features) ++b;
  return b;
}

bool compact_fits(uint32_t n_features, uint64_t max_tree_nodes) {
  const uint32_t b = compact_feature_bits(n_features);
  return (1u << b) >= n_features && max_tree_nodes <= (1ull << (32 - b));
}

int check_forest_host(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* off, uint32_t n_trees,
                      uint32_t n_features, uint32_t n_classes) {
  uint32_t bad = 0;
  for (uint32_t t = 0; t < n_trees && !bad; ++t) {
    const uint32_t b = off[t], e = t + 1 < n_trees ? off[t + 1] : n_nodes;
    if (!(b < e && e <= n_nodes)) {
      bad |= 1u;
      break;
    }
    for (uint32_t i = b; i < e; ++i) {
      const ct_packed_node& nd = nodes[i];
      if (nd.left != 0) {
        if (nd.left <= i - b || (uint64_t)nd.left + 1 >= (uint64_t)(e - b)) bad |= 2u;
        if (nd.feature >= n_features) bad |= 4u;
      } else if (nd.value >= n_classes) {
        bad |= 8u;
      }
    }
  }
  if (bad) {
    set_last_error(std::string("malformed forest: ") + forest_error_text(bad));
    return CT_ERR_ARG;
  }
  return CT_OK;
}

void compact_host(const ct_packed_node* in, uint32_t n, uint32_t fbits, ct_compact_node* out) {
  for (uint32_t i = 0; i < n; ++i) {
    const ct_packed_node& p = in[i];
    uint32_t thr;
    std::memcpy(&thr, &p.threshold, 4);
    out[i] = p.left ? ct_compact_node{thr, (p.left << fbits) | p.feature} : ct_compact_node{p.value, 0u};
  }
}

int compact_forest(const ct_packed_node* nodes, uint32_t n_nodes, uint32_t n_features, uint32_t max_tree_nodes,
                   ct_compact_node* out, cudaStream_t st) {
  CT_ARG_CHECK(nodes && out, "compact: NULL argument");
  CT_ARG_CHECK(((uintptr_t)nodes & 15u) == 0 && ((uintptr_t)out & 7u) == 0, "compact: misaligned arrays");
  CT_ARG_CHECK(n_features >= 1 && compact_fits(n_features, max_tree_nodes),
               "compact: trees too large for the compact form with this feature count");
  if (n_nodes == 0) return CT_OK;
  const uint32_t fbits = compact_feature_bits(n_features);
  k_compact<<<std::min<uint32_t>(ceil_div(n_nodes, 256), 148 * 8), 256, 0, st>>>(nodes, n_nodes, fbits,
                                                                               reinterpret_cast<uint2*>(out));
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

__global__ void __launch_bounds__(PRED_THREADS, 4)
k_predict_batch(const BatchReq* __restrict__ reqs, uint32_t n_req) {
  extern __shared__ uint32_t smem[];
  uint32_t lo = 0, hi = n_req;  // the last request whose first block is <= blockIdx.x
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (reqs[mid].block0 <= blockIdx.x) lo = mid; else hi = mid;
  }
  const BatchReq rq = reqs[lo];
  const uint32_t local = blockIdx.x - rq.block0;
  const uint32_t g = local / rq.tiles, tile = local - g * rq.tiles;
  const uint32_t t_lo = g * rq.group;
  const uint32_t n_t = min(rq.group, rq.n_trees - t_lo);
  const uint32_t rpb = rq.rpb;
  if (rq.fbits)
    tile_work<CompactForm>(rq.nodes, rq.tree_off, rq.fbits, t_lo, n_t, rq.group >= rq.n_trees, rq.x, rq.n_rows,
                           rq.n_features, rq.n_classes, rpb, tile * rpb, rq.votes, rq.pred, smem);
  else
    tile_work<PackedForm>(rq.nodes, rq.tree_off, 0, t_lo, n_t, rq.group >= rq.n_trees, rq.x, rq.n_rows,
                          rq.n_features, rq.n_classes, rpb, tile * rpb, rq.votes, rq.pred, smem);
}

// Majority vote of the rows of requests whose trees were split into groups.
__global__ void k_vote_batch(const BatchReq* __restrict__ reqs, uint32_t n_req, uint32_t total_rows) {
  const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= total_rows) return;
  uint32_t lo = 0, hi = n_req;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (reqs[mid].row0 <= row) lo = mid; else hi = mid;
  }
  const BatchReq rq = reqs[lo];
  if (rq.group >= rq.n_trees) return;  // voted in the walk kernel
  const uint32_t r = row - rq.row0;
  const uint32_t c = warp_argmax(rq.votes + (size_t)r * rq.n_classes, rq.n_classes, nullptr);
  if ((threadIdx.x & 31) == 0) rq.pred[r] = c;
}

int predict_batch(const BatchReq* reqs_dev, uint32_t n_req, uint32_t total_blocks, uint32_t total_rows,
                  size_t smem, bool any_grouped, cudaStream_t st) {
  if (n_req == 0 || total_blocks == 0) return CT_OK;
  CT_ARG_CHECK(smem <= HIST_SMEM_BYTES + X_SMEM_BYTES, "predict batch: tile shared memory too large");
  CT_TRY(allow_smem(k_predict_batch, (int)(HIST_SMEM_BYTES + X_SMEM_BYTES)));
  k_predict_batch<<<total_blocks, PRED_THREADS, smem, st>>>(reqs_dev, n_req);
  if (any_grouped) k_vote_batch<<<ceil_div(total_rows, 8), 256, 0, st>>>(reqs_dev, n_req, total_rows);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

// fbits == 0: packed nodes; else compact nodes with that many feature bits.
int predict(const void* nodes, uint32_t n_nodes, uint32_t fbits, const uint32_t* tree_off, uint32_t n_trees,
            const float* x, uint32_t n_rows, uint32_t n_features, uint32_t n_classes, uint32_t* votes,
            uint32_t* pred, cudaStream_t st) {
  CT_ARG_CHECK(nodes && tree_off && x && pred, "predict: NULL input or output");
  CT_ARG_CHECK(((uintptr_t)nodes & (fbits ? 7u : 15u)) == 0, "predict: nodes must be aligned to the node size");
  CT_ARG_CHECK(n_trees >= 1 && n_features >= 1, "predict: empty forest or no features");
  CT_ARG_CHECK(n_nodes >= n_trees, "predict: fewer nodes than trees");
  CT_ARG_CHECK(n_classes >= 1 && n_classes <= CT_MAX_CLASSES, "predict: n_classes out of range");
  CT_ARG_CHECK(!fbits || fbits == compact_feature_bits(n_features), "predict: compact form of another feature count");
  if (n_rows == 0) return CT_OK;
  if (fbits)
    CT_TRY(check_forest_device<CompactForm>(nodes, n_nodes, tree_off, n_trees, fbits, n_features, n_classes, pred, st));
  else
    CT_TRY(check_forest_device<PackedForm>(nodes, n_nodes, tree_off, n_trees, 0, n_features, n_classes, pred, st));
  const uint32_t rpb = predict_rows_per_block(n_classes, n_features);
  const uint32_t tiles = ceil_div(n_rows, rpb);
  // Tree groups need the vote table; without one every block walks all trees.
  uint32_t group = n_trees;
  if (votes && n_trees >= 16 && n_rows >= 1024)
    group = predict_group_size(n_trees, n_nodes, fbits ? CompactForm::BYTES : PackedForm::BYTES);
  const uint32_t groups = ceil_div(n_trees, group);
  const size_t smem = predict_tile_smem(rpb, n_classes, n_features);
  if (groups > 1) CT_CUDA_TRY(cudaMemsetAsync(votes, 0, (size_t)n_rows * n_classes * sizeof(uint32_t), st));
  const int most = (int)(HIST_SMEM_BYTES + X_SMEM_BYTES);
  if (fbits) {
    CT_TRY(allow_smem(k_predict<CompactForm>, most));
    k_predict<CompactForm><<<tiles * groups, PRED_THREADS, smem, st>>>(
        nodes, tree_off, n_trees, fbits, group, tiles, x, n_rows, n_features, n_classes, rpb, votes, pred);
  } else {
    CT_TRY(allow_smem(k_predict<PackedForm>, most));
    k_predict<PackedForm><<<tiles * groups, PRED_THREADS, smem, st>>>(
        nodes, tree_off, n_trees, 0, group, tiles, x, n_rows, n_features, n_classes, rpb, votes, pred);
  }
  if (groups > 1) k_vote_rows<<<ceil_div(n_rows, 8), 256, 0, st>>>(votes, n_rows, n_classes, pred);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

}  // namespace ct
