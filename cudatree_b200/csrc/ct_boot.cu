// Bootstrap: in-bag row set of a tree and the stable compaction of every
// presorted feature row onto it (reference _get_sorted_indices +
// bootstrap_fill.cu + bootstrap_reshuffle.cu, random_forest.py:113-144).
//
// The reference draws N rows with np.random.randint and keeps np.unique of
// them (random_forest.py:123-124); here draw i of tree t is
// boot_draw(boot_key(tree_key(seed, t)), i, N), and the unique set is the
// set of marked rows.  Compaction keeps the presorted order (stable), one
// warp per (piece, feature) with a decoupled look-back across pieces.
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr uint64_t ST_AGG = 1ull << 62;
constexpr uint64_t ST_INC = 2ull << 62;
constexpr uint64_t ST_FLAG = 3ull << 62;
constexpr uint64_t ST_VAL = (1ull << 62) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 20;

__global__ void k_boot_mark(uint8_t* mark, uint64_t bk, uint32_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    mark[boot_draw(bk, i, n)] = 1;
}

__global__ void k_count_marks(const uint8_t* mark, uint32_t n, uint32_t* out) {
  uint32_t c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    c += mark[i] ? 1u : 0u;
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_set_u32(uint32_t* p, uint32_t v) { *p = v; }

struct CompactArgs {
  const void* presort;
  void* out;
  const uint8_t* mark;
  uint64_t* status;      // [n_features][pieces]
  uint32_t* ticket;
  uint32_t* error;
  uint32_t n_rows;
  uint32_t n_features;
  uint32_t pieces;
  uint32_t out_stride;
};

template <typename IdxT>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_compact(CompactArgs a) {
  const uint32_t lane = lane_id();
  uint32_t ticket = 0;
  if (lane == 0) ticket = atomicAdd(a.ticket, 1u);
  ticket = __shfl_sync(FULL, ticket, 0);
  if ((uint64_t)ticket >= (uint64_t)a.pieces * a.n_features) return;
  const uint32_t f = ticket / a.pieces;
  const uint32_t j = ticket - f * a.pieces;
  const IdxT* in = reinterpret_cast<const IdxT*>(a.presort) + (size_t)f * a.n_rows;
  IdxT* out = reinterpret_cast<IdxT*>(a.out) + (size_t)f * a.out_stride;
  const uint32_t lo = j * PART_PIECE;
  uint32_t rows[PART_ROUNDS];
  unsigned kmask[PART_ROUNDS];
  uint32_t local = 0;
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    const uint32_t p = lo + r * 32 + lane;
    rows[r] = p < a.n_rows ? (uint32_t)in[p] : 0u;
  }
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    const uint32_t p = lo + r * 32 + lane;
    kmask[r] = __ballot_sync(FULL, p < a.n_rows && a.mark[rows[r]] != 0);
    local += __popc(kmask[r]);
  }
  uint64_t* col = a.status + (size_t)f * a.pieces;
  uint32_t carry = 0;
  if (lane == 0) {
    if (j == 0) {
      cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(col[0]).store(ST_INC | local,
                                                                          cuda::memory_order_release);
    } else {
      cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(col[j]).store(ST_AGG | local,
                                                                          cuda::memory_order_release);
      uint64_t acc = 0;
      uint32_t k = j - 1;
      uint32_t spins = 0;
      while (true) {
        const uint64_t w =
            cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(col[k]).load(cuda::memory_order_acquire);
        const uint64_t flag = w & ST_FLAG;
        if (flag == 0) {
          if (++spins > SPIN_LIMIT || *reinterpret_cast<volatile uint32_t*>(a.error) != 0) {
            atomicOr(a.error, DEV_ERR_TIMEOUT);
            acc = 0;
            break;
          }
          __nanosleep(64);
          continue;
        }
        acc += w & ST_VAL;
        if (flag == ST_INC || k == 0) break;
        --k;
      }
      carry = (uint32_t)acc;
      cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(col[j]).store(
          ST_INC | (uint64_t)(carry + local), cuda::memory_order_release);
    }
  }
  carry = __shfl_sync(FULL, carry, 0);
  uint32_t run = carry;
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    if ((kmask[r] >> lane) & 1u) {
      const uint32_t dst = run + __popc(kmask[r] & lt);
      if (dst < a.out_stride) out[dst] = (IdxT)rows[r];
    }
    run += __popc(kmask[r]);
  }
}

}  // namespace

size_t bootstrap_scratch_bytes(uint32_t n_rows, uint32_t n_features) {
  const size_t pieces = ceil_div(n_rows, PART_PIECE);
  return 512 + pieces * n_features * sizeof(uint64_t) + 256;
}

int bootstrap_compact(const ct_problem* p, const ct_lists* l, uint32_t slot, uint32_t tree,
                      uint32_t* n_in_dev, void* ws, size_t wsb, cudaStream_t st) {
  const uint32_t N = p->n_rows, F = p->n_features;
  CT_ARG_CHECK(slot < l->n_slots, "slot out of range");
  CT_ARG_CHECK(l->stride >= N, "list stride smaller than n_rows");
  CT_ARG_CHECK(p->presort != nullptr, "presort is NULL");
  const size_t ib = p->index_bytes;
  char* dst = reinterpret_cast<char*>(l->si0) + (size_t)slot * F * l->stride * ib;
  if (!p->bootstrap) {
    CT_CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)l->stride * ib, p->presort, (size_t)N * ib, (size_t)N * ib, F,
                                  cudaMemcpyDeviceToDevice, st));
    k_set_u32<<<1, 1, 0, st>>>(n_in_dev + slot, N);
    CT_CUDA_TRY(cudaGetLastError());
    return CT_OK;
  }
  Arena a{reinterpret_cast<char*>(ws), wsb, 0};
  uint32_t* ctr = a.take<uint32_t>(4);  // ticket, error
  const uint32_t pieces = ceil_div(N, PART_PIECE);
  uint64_t* status = a.take<uint64_t>((size_t)pieces * F);
  if (!ctr || !status) {
    set_last_error("bootstrap workspace too small");
    return CT_ERR_OOM;
  }
  uint8_t* mark = l->mark + (size_t)slot * N;
  CT_CUDA_TRY(cudaMemsetAsync(mark, 0, N, st));
  CT_CUDA_TRY(cudaMemsetAsync(ctr, 0, 4 * sizeof(uint32_t), st));
  CT_CUDA_TRY(cudaMemsetAsync(status, 0, (size_t)pieces * F * sizeof(uint64_t), st));
  CT_CUDA_TRY(cudaMemsetAsync(n_in_dev + slot, 0, sizeof(uint32_t), st));
  const uint64_t bk = boot_key(tree_key(p->seed, tree));
  const uint32_t grid = min(ceil_div(N, 256), 148u * 16u);
  k_boot_mark<<<grid, 256, 0, st>>>(mark, bk, N);
  k_count_marks<<<grid, 256, 0, st>>>(mark, N, n_in_dev + slot);
  CompactArgs ca;
  ca.presort = p->presort;
  ca.out = dst;
  ca.mark = mark;
  ca.status = status;
  ca.ticket = ctr;
  ca.error = ctr + 1;
  ca.n_rows = N;
  ca.n_features = F;
  ca.pieces = pieces;
  ca.out_stride = l->stride;
  const uint64_t warps = (uint64_t)pieces * F;
  const uint32_t blocks = (uint32_t)((warps + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK);
  if (ib == 2)
    k_compact<uint16_t><<<blocks, THREADS_PER_BLOCK, 0, st>>>(ca);
  else
    k_compact<uint32_t><<<blocks, THREADS_PER_BLOCK, 0, st>>>(ca);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

// Error word of the last bootstrap_compact call (ticket at [0], error at [1]).
uint32_t* bootstrap_error_word(void* ws) { return reinterpret_cast<uint32_t*>(ws) + 1; }

}  // namespace ct
