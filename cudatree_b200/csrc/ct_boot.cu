// Bootstrap: in-bag row set of each tree and the stable compaction of every
// presorted feature row onto it (reference _get_sorted_indices +
// bootstrap_fill.cu + bootstrap_reshuffle.cu, random_forest.py:113-144).
//
// The reference draws N rows with np.random.randint and keeps np.unique of
// them (random_forest.py:123-124); here draw i of tree t is
// boot_draw(boot_key(tree_key(seed, t)), i, N), and the unique set is the
// set of marked rows.
//
// The compaction serves up to 128 slots from one read of each presorted row.
// The in-bag marks are transposed to one word per (row, 32 slots); each
// feature's presort is cut into items of BOOT_SEG positions; a first pass
// counts every slot's in-bag entries per item, a prefix over the items gives
// each (item, slot) its output offset, and a second pass writes the items'
// entries stably into every slot.  The reference reads the presort once per
// tree, with one block per feature.
#include <algorithm>

#include <cstring>

#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr uint32_t BOOT_WARPS = 8;   // warps per CTA
constexpr uint32_t BOOT_ROUNDS = 8;  // rounds of 32 elements per warp and tile
constexpr uint32_t BOOT_TILE = BOOT_WARPS * 32 * BOOT_ROUNDS;
constexpr uint32_t BOOT_SEG = 4 * BOOT_TILE;  // positions of one work item
constexpr uint32_t BOOT_MAXW = 4;    // in-bag words per row in one launch (128 slots)

__global__ void k_boot_mark(uint8_t* mark, uint64_t seed, uint32_t tree_lo, uint32_t n) {
  const uint32_t slot = blockIdx.y;
  const uint64_t bk = boot_key(tree_key(seed, tree_lo + slot));
  uint8_t* mk = mark + (size_t)slot * n;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    mk[boot_draw(bk, i, n)] = 1;
}

__global__ void k_count_marks(const uint8_t* mark, uint32_t n, uint32_t* out) {
  const uint32_t slot = blockIdx.y;
  const uint8_t* mk = mark + (size_t)slot * n;
  uint32_t c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    c += mk[i] ? 1u : 0u;
  c = warp_sum_u32(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out + slot, c);
}

__global__ void k_set_u32(uint32_t* p, uint32_t v, uint32_t count) {
  for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) p[i] = v;
}

// inbag[r * words + w] bit b = mark of slot 32 w + b at row r.
__global__ void k_inbag_words(const uint8_t* __restrict__ mark, uint32_t n, uint32_t n_slots, uint32_t words,
                              uint32_t* __restrict__ inbag) {
  const uint64_t total = (uint64_t)n * words;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = (uint32_t)(i % words), r = (uint32_t)(i / words);
    uint32_t v = 0;
    for (uint32_t b = 0; b < 32 && w * 32 + b < n_slots; ++b)
      v |= (mark[(size_t)(w * 32 + b) * n + r] ? 1u : 0u) << b;
    inbag[i] = v;
  }
}

struct BootMulti {
  const void* src;        // [F][N] presort (or its packed copy)
  char* out;              // buffer 0 of the first slot
  const uint32_t* inbag;  // [N][words]
  uint32_t* counts;       // [F][segs][n_slots]: in-bag entries per item and slot, then their offsets
  size_t slot_elems;      // elements between slots
  uint32_t n_rows;
  uint32_t n_features;
  uint32_t n_slots;       // <= 32 * BOOT_MAXW
  uint32_t words;
  uint32_t segs;          // items per feature
  uint32_t stride;
  uint32_t row_mask;
  // Lists written: n_lists of the n_features, list_feat[k] the k-th when
  // n_lists < n_features (a fit's virtual features keep no list), else all.
  // Items run over the written lists only.
  uint32_t n_lists;
  uint8_t list_feat[64];
};
__device__ __forceinline__ uint32_t list_feature(const BootMulti& b, uint32_t k) {
  return b.n_lists < b.n_features ? b.list_feat[k] : k;
}

// Loads a round's entries and their rows' in-bag words.
template <typename IdxT>
__device__ __forceinline__ void boot_round(const BootMulti& b, const IdxT* in, uint32_t q, uint32_t lim, uint32_t& e,
                                           uint32_t (&fl)[BOOT_MAXW]) {
  e = q < lim ? (uint32_t)__ldcs(in + q) : 0u;
  const uint32_t* row = b.inbag + (size_t)(e & b.row_mask) * b.words;
#pragma unroll
  for (uint32_t w = 0; w < BOOT_MAXW; ++w) fl[w] = (q < lim && w < b.words) ? __ldg(row + w) : 0u;
}

// Pass 1: one warp per item (feature f, positions [j BOOT_SEG, (j+1) BOOT_SEG)),
// in-bag entries per slot; lane l keeps the counts of slots l, l + 32, ...
template <typename IdxT>
__global__ void __launch_bounds__(BOOT_WARPS * 32) k_boot_count(BootMulti b) {
  const uint32_t lane = lane_id();
  const uint64_t items = (uint64_t)b.n_lists * b.segs;
  const uint64_t nw = (uint64_t)gridDim.x * BOOT_WARPS;
  for (uint64_t it = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; it < items; it += nw) {
    const uint32_t k = (uint32_t)(it / b.segs), j = (uint32_t)(it - (uint64_t)k * b.segs);
    const uint32_t f = list_feature(b, k);
    const IdxT* in = reinterpret_cast<const IdxT*>(b.src) + (size_t)f * b.n_rows;
    const uint32_t lo = j * BOOT_SEG, hi = min(lo + BOOT_SEG, b.n_rows);
    uint32_t cnt[BOOT_MAXW];
#pragma unroll
    for (uint32_t w = 0; w < BOOT_MAXW; ++w) cnt[w] = 0;
    for (uint32_t q0 = lo; q0 < hi; q0 += 32 * BOOT_ROUNDS) {  // the loads of BOOT_ROUNDS rounds in flight together
      uint32_t e[BOOT_ROUNDS], fl[BOOT_ROUNDS][BOOT_MAXW];
#pragma unroll
      for (uint32_t r = 0; r < BOOT_ROUNDS; ++r) boot_round<IdxT>(b, in, q0 + r * 32 + lane, hi, e[r], fl[r]);
#pragma unroll
      for (uint32_t w = 0; w < BOOT_MAXW; ++w) {
        if (w >= b.words) break;
        const uint32_t tn = min(32u, b.n_slots - w * 32);  // live slots of this word
        for (uint32_t t = 0; t < tn; ++t) {
          uint32_t c = 0;
#pragma unroll
          for (uint32_t r = 0; r < BOOT_ROUNDS; ++r) c += __popc(__ballot_sync(FULL, (fl[r][w] >> t) & 1u));
          if (lane == t) cnt[w] += c;
        }
      }
    }
    uint32_t* out = b.counts + (size_t)it * b.n_slots;
#pragma unroll
    for (uint32_t w = 0; w < BOOT_MAXW; ++w)
      if (w * 32 + lane < b.n_slots) out[w * 32 + lane] = cnt[w];
  }
}

// Pass 2: per (feature, slot), exclusive prefix of the items' counts.
__global__ void k_boot_offsets(BootMulti b) {
  const uint64_t total = (uint64_t)b.n_lists * b.n_slots;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t f = (uint32_t)(i / b.n_slots), t = (uint32_t)(i - (uint64_t)f * b.n_slots);
    uint32_t* c = b.counts + (size_t)f * b.segs * b.n_slots + t;
    uint32_t run = 0;
    for (uint32_t j = 0; j < b.segs; ++j) {
      const uint32_t v = c[(size_t)j * b.n_slots];
      c[(size_t)j * b.n_slots] = run;
      run += v;
    }
  }
}

// Pass 3: one CTA per item.  Per tile of BOOT_TILE positions each warp takes
// BOOT_ROUNDS consecutive rounds of 32; for every slot the in-bag entries
// keep their order: item offset + tile carry + offset of the warp + rank in
// the warp.
template <typename IdxT>
__global__ void __launch_bounds__(BOOT_WARPS * 32) k_boot_write(BootMulti b) {
  __shared__ uint32_t s_cnt[32 * BOOT_MAXW][BOOT_WARPS];
  __shared__ uint32_t s_carry[32 * BOOT_MAXW];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const unsigned lt = lanemask_lt();
  const uint64_t items = (uint64_t)b.n_lists * b.segs;
  for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const uint32_t k = (uint32_t)(it / b.segs), j = (uint32_t)(it - (uint64_t)k * b.segs);
    const uint32_t f = list_feature(b, k);
    const IdxT* in = reinterpret_cast<const IdxT*>(b.src) + (size_t)f * b.n_rows;
    IdxT* out0 = reinterpret_cast<IdxT*>(b.out) + (size_t)f * b.stride;
    const uint32_t lo = j * BOOT_SEG, hi = min(lo + BOOT_SEG, b.n_rows);
    __syncthreads();  // the previous item is done with s_carry
    for (uint32_t t = threadIdx.x; t < b.n_slots; t += blockDim.x) s_carry[t] = b.counts[(size_t)it * b.n_slots + t];
    for (uint32_t base = lo; base < hi; base += BOOT_TILE) {
      const uint32_t wbase = base + warp * (32 * BOOT_ROUNDS);
      uint32_t e[BOOT_ROUNDS], fl[BOOT_ROUNDS][BOOT_MAXW];
#pragma unroll
      for (uint32_t r = 0; r < BOOT_ROUNDS; ++r) boot_round<IdxT>(b, in, wbase + r * 32 + lane, hi, e[r], fl[r]);
#pragma unroll
      for (uint32_t w = 0; w < BOOT_MAXW; ++w) {
        if (w >= b.words) break;
        const uint32_t tn = min(32u, b.n_slots - w * 32);
        for (uint32_t t = 0; t < tn; ++t) {
          uint32_t c = 0;
#pragma unroll
          for (uint32_t r = 0; r < BOOT_ROUNDS; ++r) c += __popc(__ballot_sync(FULL, (fl[r][w] >> t) & 1u));
          if (lane == 0) s_cnt[w * 32 + t][warp] = c;
        }
      }
      __syncthreads();
#pragma unroll
      for (uint32_t w = 0; w < BOOT_MAXW; ++w) {
        if (w >= b.words) break;
        for (uint32_t t = 0; t < 32; ++t) {
          const uint32_t slot = w * 32 + t;
          if (slot >= b.n_slots) break;
          uint32_t woff = 0;
#pragma unroll
          for (uint32_t k = 0; k < BOOT_WARPS; ++k) woff += k < warp ? s_cnt[slot][k] : 0u;
          IdxT* out = out0 + (size_t)slot * b.slot_elems;
          uint32_t run = s_carry[slot] + woff;
#pragma unroll
          for (uint32_t r = 0; r < BOOT_ROUNDS; ++r) {
            const bool in_bag = (fl[r][w] >> t) & 1u;
            const unsigned m = __ballot_sync(FULL, in_bag);
            if (in_bag) __stcs(out + run + __popc(m & lt), (IdxT)e[r]);
            run += __popc(m);
          }
        }
      }
      __syncthreads();  // every warp has read s_carry and s_cnt
      for (uint32_t t = threadIdx.x; t < b.n_slots; t += blockDim.x) {
        uint32_t total = 0;
#pragma unroll
        for (uint32_t k = 0; k < BOOT_WARPS; ++k) total += s_cnt[t][k];
        s_carry[t] += total;
      }
      __syncthreads();  // s_carry settled and s_cnt free for the next tile
    }
  }
}

template <typename IdxT, typename LabT>
// Feature `ident` (NONE: none) gets the rows in row order instead of its
// presort: the row list of the virtual features (View::vslot).
__global__ void k_pack_presort(const IdxT* __restrict__ in, const LabT* __restrict__ labels, IdxT* __restrict__ out,
                               uint64_t count, uint32_t shift, uint32_t n_rows, uint32_t ident, uint64_t skip) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t f = (uint32_t)(i / n_rows);
    if (f < 64 && ((skip >> f) & 1ull)) continue;  // a list nothing reads
    const uint32_t r = f == ident ? (uint32_t)(i - (uint64_t)f * n_rows) : (uint32_t)in[i];
    out[i] = (IdxT)(r | ((uint32_t)__ldg(labels + r) << shift));
  }
}

template <typename IdxT, typename LabT>
void launch_pack_presort(const ct_problem* p, void* out, uint32_t shift, uint32_t ident, uint64_t skip,
                         cudaStream_t st) {
  const uint64_t count = (uint64_t)p->n_rows * p->n_features;
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((count + 255) / 256, 148u * 16u);
  k_pack_presort<IdxT, LabT><<<blocks, 256, 0, st>>>(reinterpret_cast<const IdxT*>(p->presort),
                                                     reinterpret_cast<const LabT*>(p->labels),
                                                     reinterpret_cast<IdxT*>(out), count, shift, p->n_rows, ident,
                                                     skip);
}

struct BootLayout {
  uint32_t* words;        // [1] error word (kept for the caller's check)
  uint32_t* inbag;        // [N][ceil(slots / 32)], slots <= 32 * BOOT_MAXW per launch
  uint32_t* counts;       // [F][segs][slots]
  size_t bytes;
};

bool boot_layout(uint32_t n_rows, uint32_t n_features, uint32_t n_slots, void* ws, size_t wsb, BootLayout* L) {
  Arena a{reinterpret_cast<char*>(ws), wsb, 0};
  const uint32_t per = std::min<uint32_t>(n_slots, 32 * BOOT_MAXW);
  L->words = a.take<uint32_t>(8);
  L->inbag = a.take<uint32_t>((size_t)n_rows * ceil_div(per, 32u));
  L->counts = a.take<uint32_t>((size_t)n_features * ceil_div(n_rows, BOOT_SEG) * per);
  L->bytes = a.used + 256;
  return ws != nullptr && a.ok();
}

}  // namespace

size_t bootstrap_scratch_bytes(uint32_t n_rows, uint32_t n_features, uint32_t n_slots) {
  BootLayout L;
  boot_layout(n_rows, n_features, n_slots, nullptr, 0, &L);
  return L.bytes;
}

// Compacts slots [slot_lo, slot_lo + n_slots) for trees tree_lo...  src is the
// [F][N] presort, or its packed copy (entries row | label << s, row ids under
// row_mask).  Bit f of skip (features below 64): feature f's lists are not
// written (a fit's virtual features other than the row-list slot: nothing
// reads them).  The workspace's word [1] is an error word that the caller
// zeroes once and reads after; nothing here waits, so it stays zero.
int bootstrap_many(const ct_problem* p, const ct_lists* l, uint32_t slot_lo, uint32_t n_slots, uint32_t tree_lo,
                   const void* src, uint32_t row_mask, uint64_t skip, uint32_t* n_in_dev, void* ws, size_t wsb,
                   cudaStream_t st) {
  const uint32_t N = p->n_rows, F = p->n_features;
  CT_ARG_CHECK(n_slots >= 1 && slot_lo + n_slots <= l->n_slots, "slot out of range");
  CT_ARG_CHECK(l->stride >= N, "list stride smaller than n_rows");
  CT_ARG_CHECK(src != nullptr, "presort is NULL");
  const size_t ib = p->index_bytes;
  const size_t slot_bytes = (size_t)F * l->stride * ib;
  char* dst = reinterpret_cast<char*>(l->si0) + slot_lo * slot_bytes;
  if (!p->bootstrap) {
    for (uint32_t s = 0; s < n_slots; ++s)
      CT_CUDA_TRY(cudaMemcpy2DAsync(dst + s * slot_bytes, (size_t)l->stride * ib, src, (size_t)N * ib,
                                    (size_t)N * ib, F, cudaMemcpyDeviceToDevice, st));
    k_set_u32<<<1, 256, 0, st>>>(n_in_dev + slot_lo, N, n_slots);
    CT_CUDA_TRY(cudaGetLastError());
    return CT_OK;
  }
  BootLayout L;
  if (!boot_layout(N, F, n_slots, ws, wsb, &L)) {
    set_last_error("bootstrap workspace too small");
    return CT_ERR_OOM;
  }
  uint8_t* mark = l->mark + (size_t)slot_lo * N;
  CT_CUDA_TRY(cudaMemsetAsync(mark, 0, (size_t)n_slots * N, st));
  CT_CUDA_TRY(cudaMemsetAsync(n_in_dev + slot_lo, 0, n_slots * sizeof(uint32_t), st));
  const dim3 grid(std::min<uint32_t>(ceil_div(N, 256), 1024), n_slots);
  k_boot_mark<<<grid, 256, 0, st>>>(mark, p->seed, tree_lo, N);
  k_count_marks<<<grid, 256, 0, st>>>(mark, N, n_in_dev + slot_lo);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t segs = ceil_div(N, BOOT_SEG);
  uint32_t n_lists = 0;
  uint8_t list_feat[64] = {};
  if (skip && F <= 64) {
    for (uint32_t f = 0; f < F; ++f)
      if (!((skip >> f) & 1ull)) list_feat[n_lists++] = (uint8_t)f;
  } else {
    n_lists = F;
  }
  const uint64_t items = (uint64_t)n_lists * segs;
  for (uint32_t s0 = 0; s0 < n_slots; s0 += 32 * BOOT_MAXW) {  // at most 128 slots per pass
    const uint32_t ns = std::min<uint32_t>(n_slots - s0, 32 * BOOT_MAXW);
    const uint32_t words = ceil_div(ns, 32u);
    const uint64_t cells = (uint64_t)N * words;
    k_inbag_words<<<(uint32_t)std::min<uint64_t>((cells + 255) / 256, 148u * 16u), 256, 0, st>>>(
        mark + (size_t)s0 * N, N, ns, words, L.inbag);
    BootMulti b;
    b.src = src;
    b.out = dst + s0 * slot_bytes;
    b.inbag = L.inbag;
    b.counts = L.counts;
    b.slot_elems = (size_t)F * l->stride;
    b.n_rows = N;
    b.n_features = F;
    b.n_slots = ns;
    b.words = words;
    b.segs = segs;
    b.stride = l->stride;
    b.row_mask = row_mask;
    b.n_lists = n_lists;
    std::memcpy(b.list_feat, list_feat, sizeof(list_feat));
    const uint32_t cblocks = (uint32_t)std::min<uint64_t>((items + BOOT_WARPS - 1) / BOOT_WARPS, (uint64_t)sms * 8);
    const uint64_t pairs = (uint64_t)n_lists * ns;
    const uint32_t oblocks = (uint32_t)std::min<uint64_t>((pairs + 255) / 256, (uint64_t)sms * 8);
    const uint32_t wblocks = (uint32_t)std::min<uint64_t>(items, (uint64_t)sms * 8);
    if (ib == 2) {
      k_boot_count<uint16_t><<<cblocks, BOOT_WARPS * 32, 0, st>>>(b);
      k_boot_offsets<<<oblocks, 256, 0, st>>>(b);
      k_boot_write<uint16_t><<<wblocks, BOOT_WARPS * 32, 0, st>>>(b);
    } else {
      k_boot_count<uint32_t><<<cblocks, BOOT_WARPS * 32, 0, st>>>(b);
      k_boot_offsets<<<oblocks, 256, 0, st>>>(b);
      k_boot_write<uint32_t><<<wblocks, BOOT_WARPS * 32, 0, st>>>(b);
    }
    CT_CUDA_TRY(cudaGetLastError());
  }
  return CT_OK;
}

// The presort with each row's label above its row id (entry row | label <<
// shift), [F][N] at out; out must not overlap the presort.  Feature ident's
// list is the rows in row order; the lists of the features in skip (below 64)
// are left unwritten.
int pack_presort(const ct_problem* p, void* out, uint32_t shift, uint32_t ident, uint64_t skip, cudaStream_t st) {
  CT_ARG_CHECK(p->presort != nullptr, "presort is NULL");
  if (p->index_bytes == 2) {
    if (p->label_bytes == 1) launch_pack_presort<uint16_t, uint8_t>(p, out, shift, ident, skip, st);
    else launch_pack_presort<uint16_t, uint16_t>(p, out, shift, ident, skip, st);
  } else {
    if (p->label_bytes == 1) launch_pack_presort<uint32_t, uint8_t>(p, out, shift, ident, skip, st);
    else launch_pack_presort<uint32_t, uint16_t>(p, out, shift, ident, skip, st);
  }
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int bootstrap_compact(const ct_problem* p, const ct_lists* l, uint32_t slot, uint32_t tree, uint32_t* n_in_dev,
                      void* ws, size_t wsb, cudaStream_t st) {
  return bootstrap_many(p, l, slot, 1, tree, p->presort, 0xffffffffu, 0, n_in_dev, ws, wsb, st);
}

}  // namespace ct
