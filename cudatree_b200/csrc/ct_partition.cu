// Stable partition of index-list segments by a per-row mark byte, for every
// feature (reference scan_reshuffle, dfs_module.cu:224-307 and
// bfs_module.cu:266-377; and, with the right part dropped, the bootstrap
// compaction of bootstrap_reshuffle.cu:9-59).
//
// A segment is one node's range [0, n) in every feature list.  Left rows
// (mark != 0) keep their order at [0, nl), right rows keep theirs at
// [nl, n).  Two kernels by segment size:
//
//   k_part_small  n <= SMALL_SEG: one warp per segment loops over all
//                 features; ranks are popc of a ballot.  For n <= 16 a warp
//                 packs 32/g features per round in lane groups of width
//                 g = next_pow2(n), so tiny nodes keep the lanes busy.
//   k_part_big    n > SMALL_SEG: persistent CTAs take (feature, tile) work
//                 items of TILE elements from a ticket counter (feature-major,
//                 so a segment's tiles are consecutive tickets).  Warp counts
//                 are scanned in shared memory and the tile's carry comes from
//                 a decoupled look-back over its predecessors' status words,
//                 read 32 at a time by one warp.  Every wait is bounded: on
//                 expiry the kernel sets an error bit and returns.
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr uint64_t ST_AGG = 1ull << 62;
constexpr uint64_t ST_INC = 2ull << 62;
constexpr uint64_t ST_FLAG = 3ull << 62;
constexpr uint64_t ST_VAL = (1ull << 62) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 20;
constexpr int BIG_WARPS = TILE_ELEMS / (32 * PART_ROUNDS);
constexpr int BIG_THREADS = BIG_WARPS * 32;
constexpr int SMALL_THREADS = 256;
constexpr uint32_t FEAT_BLOCK = 8;

__device__ __forceinline__ uint32_t read_word(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ uint32_t live(const PartWork& w, const uint32_t* count, uint32_t cap) {
  return read_word(w.error) ? 0u : min(read_word(count), cap);
}
__device__ __forceinline__ void publish(uint64_t* p, uint64_t v) {
  cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(*p).store(v, cuda::memory_order_release);
}
__device__ __forceinline__ uint64_t poll(uint64_t* p) {
  return cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(*p).load(cuda::memory_order_acquire);
}
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(FULL, v, s);
  return v;
}

// Sum of the counts of tiles [0, j) of one segment column: warp-collective
// look-back over windows of 32 predecessors.  Returns 0 and flags an error
// if a predecessor never publishes.
__device__ uint32_t window_lookback(uint64_t* col, uint32_t j, uint32_t* error) {
  const uint32_t lane = lane_id();
  uint64_t acc = 0;
  int64_t hi = (int64_t)j - 1;
  uint32_t spins = 0;
  while (true) {
    const int64_t k = hi - (int64_t)lane;
    const uint64_t word = k >= 0 ? poll(col + k) : ST_INC;
    const uint64_t flag = word & ST_FLAG;
    const unsigned inc = __ballot_sync(FULL, flag == ST_INC);
    const unsigned not_ready = __ballot_sync(FULL, flag == 0);
    const unsigned upto = inc ? (((inc & (0u - inc)) << 1) - 1u) : FULL;
    if (not_ready & upto) {
      if (++spins > SPIN_LIMIT || read_word(error) != 0) {
        if (lane == 0) atomicOr(error, DEV_ERR_TIMEOUT);
        return 0;
      }
      __nanosleep(32);
      continue;
    }
    acc += warp_sum_u64(((upto >> lane) & 1u) ? (word & ST_VAL) : 0ull);
    if (inc) break;
    hi -= 32;
  }
  return (uint32_t)acc;
}

// One warp per (segment, block of FEAT_BLOCK features).  Segments of up to
// 16 rows pack 32/g features per round in lane groups of width g; larger ones
// take one feature per pass of up to PART_ROUNDS rounds.  Loads of the
// block's rounds are issued before their marks are read, so a warp keeps
// several independent index->mark chains in flight.
template <typename IdxT>
__global__ void __launch_bounds__(SMALL_THREADS, 4) k_part_small(PartWork w) {
  const uint32_t lane = lane_id();
  const uint32_t nseg = live(w, w.n_small, w.cap_small);
  const uint32_t F = w.n_features;
  const uint32_t nfb = ceil_div(F, FEAT_BLOCK);
  const uint64_t items = (uint64_t)nseg * nfb;
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const unsigned lt = lanemask_lt();
  for (uint64_t it = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; it < items; it += nwarps) {
    const uint32_t si = (uint32_t)(it / nfb);
    const uint32_t f_lo = (uint32_t)(it - (uint64_t)si * nfb) * FEAT_BLOCK;
    const uint32_t f_hi = min(f_lo + FEAT_BLOCK, F);
    const PartSeg sg = w.small[si];
    const IdxT* in = reinterpret_cast<const IdxT*>(sg.in);
    IdxT* out = reinterpret_cast<IdxT*>(sg.out);
    const uint32_t n = sg.n, nl = sg.nl;
    if (n <= 16) {
      uint32_t g = 1;
      while (g < n) g <<= 1;
      const uint32_t per = 32 / g, sub = lane / g, p = lane & (g - 1);
      const unsigned gmask = ((g == 32) ? FULL : ((1u << g) - 1u)) << (sub * g);
      constexpr uint32_t R = FEAT_BLOCK;  // rounds needed when g == 32 / per == 1 (never for n <= 16)
      uint32_t rows[R];
      bool valid[R];
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        const uint32_t f = f_lo + r * per + sub;
        valid[r] = f < f_hi && p < n;
        rows[r] = valid[r] ? (uint32_t)in[(size_t)f * sg.in_fstride + p] : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        if (f_lo + r * per >= f_hi) break;
        const uint32_t f = f_lo + r * per + sub;
        const bool left = valid[r] && sg.mark[rows[r]] != 0;
        const unsigned lm = __ballot_sync(FULL, left) & gmask;
        const uint32_t rl = __popc(lm & lt);
        const uint32_t dst = left ? rl : nl + (p - rl);
        if (valid[r] && (left || sg.keep_right) && dst < n)
          out[(size_t)f * sg.out_fstride + dst] = (IdxT)rows[r];
      }
    } else if (n <= 32) {
      uint32_t rows[FEAT_BLOCK];
#pragma unroll
      for (uint32_t r = 0; r < FEAT_BLOCK; ++r) {
        const uint32_t f = f_lo + r;
        rows[r] = (f < f_hi && lane < n) ? (uint32_t)in[(size_t)f * sg.in_fstride + lane] : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < FEAT_BLOCK; ++r) {
        const uint32_t f = f_lo + r;
        if (f >= f_hi) break;
        const bool valid = lane < n;
        const bool left = valid && sg.mark[rows[r]] != 0;
        const unsigned lm = __ballot_sync(FULL, left);
        const uint32_t rl = __popc(lm & lt);
        const uint32_t dst = left ? rl : nl + (lane - rl);
        if (valid && (left || sg.keep_right) && dst < n) out[(size_t)f * sg.out_fstride + dst] = (IdxT)rows[r];
      }
    } else {
      const uint32_t rounds = ceil_div(n, 32);
      for (uint32_t f = f_lo; f < f_hi; ++f) {
        const IdxT* fin = in + (size_t)f * sg.in_fstride;
        IdxT* fout = out + (size_t)f * sg.out_fstride;
        uint32_t rows[PART_ROUNDS];
#pragma unroll
        for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
          const uint32_t p = r * 32 + lane;
          rows[r] = (r < rounds && p < n) ? (uint32_t)fin[p] : 0u;
        }
        uint32_t run = 0;
#pragma unroll
        for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
          if (r >= rounds) break;
          const uint32_t p = r * 32 + lane;
          const bool valid = p < n;
          const bool left = valid && sg.mark[rows[r]] != 0;
          const unsigned lm = __ballot_sync(FULL, left);
          const uint32_t rl = run + __popc(lm & lt);
          const uint32_t dst = left ? rl : nl + (p - rl);
          if (valid && (left || sg.keep_right) && dst < n) fout[dst] = (IdxT)rows[r];
          run += __popc(lm);
        }
      }
    }
  }
}

// ---- TMA bulk copies (cp.async.bulk, 1-D) with mbarrier completion --------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Global -> shared bulk copy; src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// One claimed (tile, feature) work item of k_part_big.
struct TileJob {
  const void* src16;      // 16-byte aligned start of the copied range
  void* out;              // feature f's output base of the segment
  const uint8_t* mark;
  uint64_t* col;          // status column of (segment, feature)
  uint32_t bytes;         // copied bytes (multiple of 16)
  uint32_t off;           // element offset of the tile inside the copied range
  uint32_t lo;            // first segment position of the tile
  uint32_t cnt;           // elements in the tile
  uint32_t n, nl, j, ntiles, keep_right, valid;
};

template <typename IdxT>
__device__ __forceinline__ void claim_tile(const PartWork& w, uint32_t ntiles, uint64_t tasks, TileJob* jb) {
  const uint32_t t = atomicAdd(w.ticket, 1u);
  if ((uint64_t)t >= tasks) {
    jb->valid = 0;
    return;
  }
  // tile-major: the predecessor (k-1, f) of a tile was issued n_features
  // tickets earlier, so its status is usually published by the time we look
  const uint32_t k = t / w.n_features;
  const uint32_t f = t - k * w.n_features;
  const PartTile tl = w.tiles[k];
  const PartSeg sg = w.big[tl.seg];
  const uint32_t lo = tl.j * TILE_ELEMS;
  const uint32_t cnt = min(TILE_ELEMS, sg.n - lo);
  const IdxT* src = reinterpret_cast<const IdxT*>(sg.in) + (size_t)f * sg.in_fstride + lo;
  const uintptr_t a = reinterpret_cast<uintptr_t>(src);
  const uintptr_t a0 = a & ~uintptr_t(15);
  const uintptr_t e1 = (a + (uintptr_t)cnt * sizeof(IdxT) + 15) & ~uintptr_t(15);
  jb->src16 = reinterpret_cast<const void*>(a0);
  jb->bytes = (uint32_t)(e1 - a0);
  jb->off = (uint32_t)((a - a0) / sizeof(IdxT));
  jb->out = reinterpret_cast<IdxT*>(sg.out) + (size_t)f * sg.out_fstride;
  jb->mark = sg.mark;
  jb->col = w.status + (size_t)f * w.cap_status + sg.status;
  jb->lo = lo;
  jb->cnt = cnt;
  jb->n = sg.n;
  jb->nl = sg.nl;
  jb->j = tl.j;
  jb->ntiles = tl.ntiles;
  jb->keep_right = sg.keep_right;
  jb->valid = 1;
}

// Persistent CTAs; the index tile of the next ticket is brought into shared
// memory by a TMA bulk copy while the current tile gathers its marks, looks
// back for its carry and stores.  Copies read up to 15 bytes past a tile's
// last element (16-byte rounding); list buffers carry that padding.
template <typename IdxT>
__global__ void __launch_bounds__(BIG_THREADS) k_part_big(PartWork w) {
  constexpr uint32_t BUF = TILE_ELEMS * sizeof(IdxT) + 32;
  __shared__ alignas(128) unsigned char sbuf[2][BUF];
  __shared__ alignas(8) uint64_t bars[2];
  __shared__ TileJob jobs[2];
  __shared__ uint32_t s_carry;
  __shared__ uint32_t s_wcnt[BIG_WARPS], s_woff[BIG_WARPS];
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  const uint32_t ntiles = live(w, w.n_tiles, w.cap_tiles);
  const uint64_t tasks = (uint64_t)ntiles * w.n_features;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
    claim_tile<IdxT>(w, ntiles, tasks, &jobs[0]);
    if (jobs[0].valid) {
      mbar_expect_tx(&bars[0], jobs[0].bytes);
      bulk_g2s(sbuf[0], jobs[0].src16, jobs[0].bytes, &bars[0]);
    }
  }
  __syncthreads();
  uint32_t phase[2] = {0u, 0u};
  for (uint32_t it = 0;; ++it) {
    const uint32_t b = it & 1u;
    if (!jobs[b].valid) break;
    if (threadIdx.x == 0) {  // prefetch the next work item into the other buffer
      claim_tile<IdxT>(w, ntiles, tasks, &jobs[b ^ 1u]);
      if (jobs[b ^ 1u].valid) {
        mbar_expect_tx(&bars[b ^ 1u], jobs[b ^ 1u].bytes);
        bulk_g2s(sbuf[b ^ 1u], jobs[b ^ 1u].src16, jobs[b ^ 1u].bytes, &bars[b ^ 1u]);
      }
    }
    // wait for this tile's indices (bounded; a copy of at most 16 KiB)
    bool ok = true;
    {
      uint32_t spins = 0;
      while (!mbar_try_wait(&bars[b], phase[b])) {
        if (++spins > (SPIN_LIMIT << 2)) {
          ok = false;
          break;
        }
      }
    }
    if (!__syncthreads_and(ok)) {
      // never read a tile that did not arrive: flag, drain both buffers' copies (bounded), leave
      if (threadIdx.x == 0) atomicOr(w.error, DEV_ERR_TIMEOUT);
      uint32_t spins = 0;
      while (!mbar_try_wait(&bars[b], phase[b]) && ++spins < (SPIN_LIMIT << 4)) {
      }
      if (jobs[b ^ 1u].valid) {
        spins = 0;
        while (!mbar_try_wait(&bars[b ^ 1u], phase[b ^ 1u]) && ++spins < (SPIN_LIMIT << 4)) {
        }
      }
      return;
    }
    phase[b] ^= 1u;
    const TileJob jb = jobs[b];
    const IdxT* rows = reinterpret_cast<const IdxT*>(sbuf[b]) + jb.off;
    const uint32_t wlo = warp * (32 * PART_ROUNDS);
    unsigned lmask[PART_ROUNDS];
    uint32_t cnt = 0;
#pragma unroll
    for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
      const uint32_t q = wlo + r * 32 + lane;
      const bool left = q < jb.cnt && jb.mark[(uint32_t)rows[q < jb.cnt ? q : 0]] != 0;
      lmask[r] = __ballot_sync(FULL, left);
      cnt += __popc(lmask[r]);
    }
    if (lane == 0) s_wcnt[warp] = cnt;
    __syncthreads();
    if (warp == 0) {
      const uint32_t c = lane < BIG_WARPS ? s_wcnt[lane] : 0u;
      uint32_t inc = c;
#pragma unroll
      for (int sft = 1; sft < BIG_WARPS; sft <<= 1) {
        const uint32_t o = __shfl_up_sync(FULL, inc, sft);
        if (lane >= (uint32_t)sft) inc += o;
      }
      if (lane < BIG_WARPS) s_woff[lane] = inc - c;
      const uint32_t total = __shfl_sync(FULL, inc, BIG_WARPS - 1);
      uint32_t carry = 0;
      if (jb.ntiles > 1) {
        if (jb.j == 0) {
          if (lane == 0) publish(jb.col, ST_INC | total);
        } else {
          if (lane == 0) publish(jb.col + jb.j, ST_AGG | total);
          carry = window_lookback(jb.col, jb.j, w.error);
          if (lane == 0) publish(jb.col + jb.j, ST_INC | (uint64_t)(carry + total));
        }
      }
      if (lane == 0) s_carry = carry;
    }
    __syncthreads();
    uint32_t run = s_carry + s_woff[warp];
    IdxT* out = reinterpret_cast<IdxT*>(jb.out);
#pragma unroll
    for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
      const uint32_t q = wlo + r * 32 + lane;
      const bool left = (lmask[r] >> lane) & 1u;
      const uint32_t rl = run + __popc(lmask[r] & lt);
      if (q < jb.cnt && (left || jb.keep_right)) {
        const uint32_t p = jb.lo + q;
        const uint32_t dst = left ? rl : jb.nl + (p - rl);
        if (dst < jb.n) out[dst] = rows[q];
      }
      run += __popc(lmask[r]);
    }
    __syncthreads();
  }
}

template <typename K>
int resident_blocks(K kernel, int threads) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
  return sms * (per > 0 ? per : 1);
}

}  // namespace

int launch_seg_partition(uint32_t index_bytes, const PartWork& w, uint64_t bound_small, uint64_t bound_tiles,
                         cudaStream_t st) {
  if (bound_small > 0) {
    const uint64_t items = bound_small * ceil_div(w.n_features, FEAT_BLOCK);
    const uint64_t want = (items + (SMALL_THREADS / 32) - 1) / (SMALL_THREADS / 32);
    if (index_bytes == 2) {
      const int cap = resident_blocks(k_part_small<uint16_t>, SMALL_THREADS);
      k_part_small<uint16_t><<<(uint32_t)std::min<uint64_t>(want, cap), SMALL_THREADS, 0, st>>>(w);
    } else {
      const int cap = resident_blocks(k_part_small<uint32_t>, SMALL_THREADS);
      k_part_small<uint32_t><<<(uint32_t)std::min<uint64_t>(want, cap), SMALL_THREADS, 0, st>>>(w);
    }
  }
  if (bound_tiles > 0) {
    const uint64_t want = bound_tiles * w.n_features;
    if (index_bytes == 2) {
      const int cap = resident_blocks(k_part_big<uint16_t>, BIG_THREADS);
      k_part_big<uint16_t><<<(uint32_t)std::min<uint64_t>(want, cap), BIG_THREADS, 0, st>>>(w);
    } else {
      const int cap = resident_blocks(k_part_big<uint32_t>, BIG_THREADS);
      k_part_big<uint32_t><<<(uint32_t)std::min<uint64_t>(want, cap), BIG_THREADS, 0, st>>>(w);
    }
  }
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

}  // namespace ct
