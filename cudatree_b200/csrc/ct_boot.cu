// Bootstrap: in-bag row set of each tree and the stable compaction of every
// presorted feature row onto it (reference _get_sorted_indices +
// bootstrap_fill.cu + bootstrap_reshuffle.cu, random_forest.py:113-144).
//
// The reference draws N rows with np.random.randint and keeps np.unique of
// them (random_forest.py:123-124); here draw i of tree t is
// boot_draw(boot_key(tree_key(seed, t)), i, N), and the unique set is the
// set of marked rows.  The compaction is the tiled stable partition of
// ct_partition.cu with the right (out-of-bag) part dropped; all slots of a
// call are compacted by one launch.
#include <algorithm>

#include "ct_internal.cuh"

namespace ct {

namespace {

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

template <typename IdxT, typename LabT>
__global__ void k_pack_presort(const IdxT* __restrict__ in, const LabT* __restrict__ labels, IdxT* __restrict__ out,
                               uint64_t count, uint32_t shift) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = in[i];
    out[i] = (IdxT)(r | ((uint32_t)__ldg(labels + r) << shift));
  }
}

template <typename IdxT, typename LabT>
void launch_pack_presort(const ct_problem* p, void* out, uint32_t shift, cudaStream_t st) {
  const uint64_t count = (uint64_t)p->n_rows * p->n_features;
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((count + 255) / 256, 148u * 16u);
  k_pack_presort<IdxT, LabT><<<blocks, 256, 0, st>>>(reinterpret_cast<const IdxT*>(p->presort),
                                                     reinterpret_cast<const LabT*>(p->labels),
                                                     reinterpret_cast<IdxT*>(out), count, shift);
}

struct BootPlan {
  const void* presort;
  char* si0;              // slot 0 of buffer 0
  const uint32_t* bits;   // slot 0 packed mark table
  PartSeg* segs;
  PartTile* tiles;
  size_t slot_bytes;      // bytes between slots in si0
  uint32_t n_rows;
  uint32_t stride;
  uint32_t tiles_per_slot;
};

__global__ void k_boot_plan(BootPlan b) {
  const uint32_t slot = blockIdx.x;
  if (threadIdx.x == 0) {
    PartSeg sg;
    sg.in = b.presort;
    sg.out = b.si0 + slot * b.slot_bytes;
    sg.bits = b.bits + (size_t)slot * mark_bit_words(b.n_rows);
    sg.in_fstride = b.n_rows;
    sg.out_fstride = b.stride;
    sg.n = b.n_rows;
    sg.nl = 0;
    sg.keep_right = 0;
    sg.status = slot * b.tiles_per_slot;
    b.segs[slot] = sg;
  }
  for (uint32_t j = threadIdx.x; j < b.tiles_per_slot; j += blockDim.x) {
    PartTile tl;
    tl.seg = slot;
    tl.j = j;
    tl.ntiles = b.tiles_per_slot;
    tl.pad = 0;
    b.tiles[(size_t)slot * b.tiles_per_slot + j] = tl;
  }
}

struct BootLayout {
  uint32_t* words;        // [0] ticket, [1] error, [2] n_big, [3] n_tiles, [4] n_small
  PartSeg* segs;
  PartTile* tiles;
  uint64_t* status;
  size_t bytes;
};

bool boot_layout(uint32_t n_rows, uint32_t n_features, uint32_t n_slots, void* ws, size_t wsb, BootLayout* L) {
  Arena a{reinterpret_cast<char*>(ws), wsb, 0};
  const size_t tiles = (size_t)ceil_div(n_rows, TILE_ELEMS) * n_slots;
  L->words = a.take<uint32_t>(8);
  L->segs = a.take<PartSeg>(n_slots);
  L->tiles = a.take<PartTile>(tiles);
  L->status = a.take<uint64_t>(tiles * n_features);
  L->bytes = a.used + 256;
  return ws != nullptr && a.ok();
}

}  // namespace

size_t bootstrap_scratch_bytes(uint32_t n_rows, uint32_t n_features, uint32_t n_slots) {
  BootLayout L;
  boot_layout(n_rows, n_features, n_slots, nullptr, 0, &L);
  return L.bytes;
}

// Compacts slots [slot_lo, slot_lo + n_slots) for trees tree_lo.., one launch
// per phase.  src is the [F][N] presort, or its packed copy (entries
// row | label << s, row ids under row_mask).  Error bits accumulate in the
// workspace's word [1]; the caller zeroes it once and reads it after.
int bootstrap_many(const ct_problem* p, const ct_lists* l, uint32_t slot_lo, uint32_t n_slots, uint32_t tree_lo,
                   const void* src, uint32_t row_mask, uint32_t* n_in_dev, void* ws, size_t wsb,
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
  const uint32_t tiles_per = ceil_div(N, TILE_ELEMS);
  uint8_t* mark = l->mark + (size_t)slot_lo * N;
  CT_CUDA_TRY(cudaMemsetAsync(mark, 0, (size_t)n_slots * N, st));
  CT_CUDA_TRY(cudaMemsetAsync(L.words, 0, sizeof(uint32_t), st));  // ticket (error word kept)
  CT_CUDA_TRY(cudaMemsetAsync(n_in_dev + slot_lo, 0, n_slots * sizeof(uint32_t), st));
  uint32_t counts[3] = {n_slots, tiles_per * n_slots, 0};
  k_set_u32<<<1, 32, 0, st>>>(L.words + 2, counts[0], 1);
  k_set_u32<<<1, 32, 0, st>>>(L.words + 3, counts[1], 1);
  k_set_u32<<<1, 32, 0, st>>>(L.words + 4, 0, 1);
  const dim3 grid(std::min<uint32_t>(ceil_div(N, 256), 1024), n_slots);
  k_boot_mark<<<grid, 256, 0, st>>>(mark, p->seed, tree_lo, N);
  k_count_marks<<<grid, 256, 0, st>>>(mark, N, n_in_dev + slot_lo);
  uint32_t* bits = reinterpret_cast<uint32_t*>(l->mark + mark_bits_offset(N, l->n_slots)) +
                   (size_t)slot_lo * mark_bit_words(N);
  launch_pack_marks(mark, bits, N, n_slots, st);
  BootPlan b;
  b.presort = src;
  b.si0 = dst;
  b.bits = bits;
  b.segs = L.segs;
  b.tiles = L.tiles;
  b.slot_bytes = slot_bytes;
  b.n_rows = N;
  b.stride = l->stride;
  b.tiles_per_slot = tiles_per;
  k_boot_plan<<<n_slots, 128, 0, st>>>(b);
  CT_CUDA_TRY(cudaGetLastError());
  PartWork w;
  w.small = nullptr;
  w.n_small = L.words + 4;
  w.cap_small = 0;
  w.big = L.segs;
  w.n_big = L.words + 2;
  w.cap_big = n_slots;
  w.tiles = L.tiles;
  w.n_tiles = L.words + 3;
  w.cap_tiles = tiles_per * n_slots;
  w.status = L.status;
  w.cap_status = tiles_per * n_slots;
  w.ticket = L.words;
  w.error = L.words + 1;
  w.n_features = F;
  w.row_mask = row_mask;
  return launch_seg_partition((uint32_t)ib, w, 0, (uint64_t)tiles_per * n_slots, st);
}

// The presort with each row's label above its row id (entry row | label <<
// shift), [F][N] at out; out must not overlap the presort.
int pack_presort(const ct_problem* p, void* out, uint32_t shift, cudaStream_t st) {
  CT_ARG_CHECK(p->presort != nullptr, "presort is NULL");
  if (p->index_bytes == 2) {
    if (p->label_bytes == 1) launch_pack_presort<uint16_t, uint8_t>(p, out, shift, st);
    else launch_pack_presort<uint16_t, uint16_t>(p, out, shift, st);
  } else {
    if (p->label_bytes == 1) launch_pack_presort<uint32_t, uint8_t>(p, out, shift, st);
    else launch_pack_presort<uint32_t, uint16_t>(p, out, shift, st);
  }
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int bootstrap_compact(const ct_problem* p, const ct_lists* l, uint32_t slot, uint32_t tree, uint32_t* n_in_dev,
                      void* ws, size_t wsb, cudaStream_t st) {
  return bootstrap_many(p, l, slot, 1, tree, p->presort, 0xffffffffu, n_in_dev, ws, wsb, st);
}

}  // namespace ct
