// Forest prediction: tree traversal + device-side majority vote.
//
// Reference: predict.cu:12-69 walks one tree per launch with one active lane
// per warp, and random_forest.py:339-362 stacks per-tree labels on the host
// and votes row by row in Python.  Here one launch walks every tree of the
// packed forest for a tile of rows: the rows are staged in shared memory,
// each thread walks several (row, tree) pairs interleaved so their node
// loads overlap, and votes accumulate in a shared-memory histogram.  The
// winner is the class with most votes, lowest class id on ties
// (np.argmax(np.bincount(...)), random_forest.py:358).
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr int PRED_THREADS = 256;
constexpr int PRED_ILP = 4;

__global__ void __launch_bounds__(PRED_THREADS)
k_predict(const ct_packed_node* __restrict__ nodes, const uint32_t* __restrict__ tree_off, uint32_t n_trees,
          const float* __restrict__ x, uint32_t n_rows, uint32_t n_features, uint32_t n_classes,
          uint32_t rows_per_block, uint32_t x_in_smem, uint32_t* __restrict__ votes,
          uint32_t* __restrict__ pred) {
  extern __shared__ uint32_t smem[];
  uint32_t* hist = smem;                                            // [rows_per_block][C]
  float* xs = reinterpret_cast<float*>(smem + rows_per_block * n_classes);  // [rows][F]
  const uint32_t row0 = blockIdx.x * rows_per_block;
  const uint32_t rows = min(rows_per_block, n_rows - row0);
  for (uint32_t i = threadIdx.x; i < rows_per_block * n_classes; i += blockDim.x) hist[i] = 0;
  if (x_in_smem)
    for (uint32_t i = threadIdx.x; i < rows * n_features; i += blockDim.x)
      xs[i] = x[(size_t)row0 * n_features + i];
  __syncthreads();
  const uint64_t work = (uint64_t)rows * n_trees;
  for (uint64_t w0 = (uint64_t)threadIdx.x * PRED_ILP; w0 < work; w0 += (uint64_t)blockDim.x * PRED_ILP) {
    uint32_t idx[PRED_ILP], base[PRED_ILP], r[PRED_ILP];
    bool live[PRED_ILP];
#pragma unroll
    for (int k = 0; k < PRED_ILP; ++k) {
      const uint64_t w = w0 + k;
      live[k] = w < work;
      r[k] = live[k] ? (uint32_t)(w / n_trees) : 0;
      const uint32_t t = live[k] ? (uint32_t)(w - (uint64_t)r[k] * n_trees) : 0;
      base[k] = tree_off[t];
      idx[k] = 0;
    }
    bool any = true;
    while (any) {
      any = false;
#pragma unroll
      for (int k = 0; k < PRED_ILP; ++k) {
        if (!live[k]) continue;
        const ct_packed_node nd = nodes[base[k] + idx[k]];
        if (nd.left == 0) {
          atomicAdd(&hist[r[k] * n_classes + nd.value], 1u);
          live[k] = false;
          continue;
        }
        const float xv = x_in_smem ? xs[r[k] * n_features + nd.feature]
                                   : x[(size_t)(row0 + r[k]) * n_features + nd.feature];
        idx[k] = (xv < nd.threshold) ? nd.left : nd.left + 1;
        any = true;
      }
    }
  }
  __syncthreads();
  // one warp per row: argmax with lowest class on ties
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t rr = warp; rr < rows; rr += blockDim.x >> 5) {
    uint32_t best = 0, bc = NONE;
    for (uint32_t c = lane; c < n_classes; c += 32) {
      const uint32_t v = hist[rr * n_classes + c];
      if (votes) votes[(size_t)(row0 + rr) * n_classes + c] = v;
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
    if (lane == 0 && pred) pred[row0 + rr] = bc;
  }
}

// One request of a batched predict launch.
}  // namespace

__global__ void __launch_bounds__(PRED_THREADS)
k_predict_batch(const BatchReq* __restrict__ reqs, uint32_t n_req, uint32_t rows_per_block) {
  extern __shared__ uint32_t smem[];
  // request of this block: the last request whose first block is <= blockIdx.x
  uint32_t lo = 0, hi = n_req;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (reqs[mid].block0 <= blockIdx.x) lo = mid; else hi = mid;
  }
  const BatchReq rq = reqs[lo];
  const uint32_t n_classes = rq.n_classes, n_features = rq.n_features, n_trees = rq.n_trees;
  uint32_t* hist = smem;
  const uint32_t row0 = (blockIdx.x - rq.block0) * rows_per_block;
  const uint32_t rows = min(rows_per_block, rq.n_rows - row0);
  for (uint32_t i = threadIdx.x; i < rows_per_block * n_classes; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const float* x = rq.x + (size_t)row0 * n_features;
  const ct_packed_node* __restrict__ nodes = rq.nodes;
  const uint64_t work = (uint64_t)rows * n_trees;
  for (uint64_t w0 = (uint64_t)threadIdx.x * PRED_ILP; w0 < work; w0 += (uint64_t)blockDim.x * PRED_ILP) {
    uint32_t idx[PRED_ILP], base[PRED_ILP], r[PRED_ILP];
    bool live[PRED_ILP];
#pragma unroll
    for (int k = 0; k < PRED_ILP; ++k) {
      const uint64_t w = w0 + k;
      live[k] = w < work;
      r[k] = live[k] ? (uint32_t)(w / n_trees) : 0;
      const uint32_t t = live[k] ? (uint32_t)(w - (uint64_t)r[k] * n_trees) : 0;
      base[k] = rq.tree_off[t];
      idx[k] = 0;
    }
    bool any = true;
    while (any) {
      any = false;
#pragma unroll
      for (int k = 0; k < PRED_ILP; ++k) {
        if (!live[k]) continue;
        const ct_packed_node nd = nodes[base[k] + idx[k]];
        if (nd.left == 0) {
          atomicAdd(&hist[r[k] * n_classes + nd.value], 1u);
          live[k] = false;
          continue;
        }
        idx[k] = (__ldg(x + (size_t)r[k] * n_features + nd.feature) < nd.threshold) ? nd.left : nd.left + 1;
        any = true;
      }
    }
  }
  __syncthreads();
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t rr = warp; rr < rows; rr += blockDim.x >> 5) {
    uint32_t best = 0, bc = NONE;
    for (uint32_t c = lane; c < n_classes; c += 32) {
      const uint32_t v = hist[rr * n_classes + c];
      if (bc == NONE || v > best) {
        best = v;
        bc = c;
      }
    }
#pragma unroll
    for (int s2 = 16; s2 > 0; s2 >>= 1) {
      const uint32_t ob = __shfl_xor_sync(FULL, best, s2);
      const uint32_t oc = __shfl_xor_sync(FULL, bc, s2);
      if (oc != NONE && (bc == NONE || ob > best || (ob == best && oc < bc))) {
        best = ob;
        bc = oc;
      }
    }
    if (lane == 0) rq.pred[row0 + rr] = bc;
  }
}

int predict_batch(const BatchReq* reqs_dev, uint32_t n_req, uint32_t total_blocks, uint32_t rows_per_block,
                  uint32_t max_classes, cudaStream_t st) {
  if (n_req == 0 || total_blocks == 0) return CT_OK;
  const size_t smem = (size_t)rows_per_block * max_classes * sizeof(uint32_t);
  k_predict_batch<<<total_blocks, PRED_THREADS, smem, st>>>(reqs_dev, n_req, rows_per_block);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int predict(const ct_packed_node* nodes, const uint32_t* tree_off, uint32_t n_trees, const float* x,
            uint32_t n_rows, uint32_t n_features, uint32_t n_classes, uint32_t* votes, uint32_t* pred,
            cudaStream_t st) {
  CT_ARG_CHECK(nodes && tree_off && x, "predict: NULL input");
  CT_ARG_CHECK(n_trees >= 1 && n_features >= 1, "predict: empty forest or no features");
  CT_ARG_CHECK(n_classes >= 1 && n_classes <= CT_MAX_CLASSES, "predict: n_classes out of range");
  if (n_rows == 0) return CT_OK;
  uint32_t rpb = 8;
  size_t hist_bytes = (size_t)rpb * n_classes * sizeof(uint32_t);
  size_t x_bytes = (size_t)rpb * n_features * sizeof(float);
  uint32_t x_in_smem = (hist_bytes + x_bytes) <= 48 * 1024 ? 1u : 0u;
  const size_t smem = hist_bytes + (x_in_smem ? x_bytes : 0);
  const uint32_t blocks = ceil_div(n_rows, rpb);
  k_predict<<<blocks, PRED_THREADS, smem, st>>>(nodes, tree_off, n_trees, x, n_rows, n_features, n_classes, rpb,
                                                x_in_smem, votes, pred);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

}  // namespace ct
