// Stable partition of index-list segments by a per-row mark bit, for every
// feature (reference scan_reshuffle, dfs_module.cu:224-307 and
// bfs_module.cu:266-377).
//
// A segment is one node's range [0, n) in every feature list.  Left rows
// (mark != 0) keep their order at [0, nl), right rows keep theirs at
// [nl, n).  Entries move unchanged; an entry's row id (its mark bit) is
// entry & row_mask, since fit lists carry the label above the row id.
// Two kernels by segment size:
//
//   k_part_small  n <= small_rows (ct_fit_options, default SMALL_SEG): one
//                 warp per segment loops over all
//                 features; ranks are popc of a ballot.  For n <= 16 a warp
//                 packs 32/g features per round in lane groups of width
//                 g = next_pow2(n), so tiny nodes keep the lanes busy.
//   k_part_big    larger n: persistent CTAs claim whole (segment,
//                 feature) chains from a ticket counter and stream the chain's
//                 tiles of TILE elements in order through a ring of shared-
//                 memory buffers filled by TMA bulk copies; the running left
//                 count is a register, so no CTA waits for another.  Every
//                 wait on a copy is bounded: on expiry the kernel sets an
//                 error bit, drains its copies and returns.
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr uint32_t SPIN_LIMIT = 1u << 20;
constexpr int BIG_WARPS = 8;  // warps of a k_part_big CTA
constexpr int BIG_THREADS = BIG_WARPS * 32;
constexpr int SMALL_THREADS = 256;
constexpr uint32_t FEAT_BLOCK = 8;

__device__ __forceinline__ uint32_t read_word(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ uint32_t live(const PartWork& w, const uint32_t* count, uint32_t cap) {
  return read_word(w.error) ? 0u : min(read_word(count), cap);
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
    const PartSeg sg = w.small[si];
    if (f_lo >= sg.n_features) continue;  // a job of fewer features than the batch's most
    const uint32_t f_hi = min(f_lo + FEAT_BLOCK, sg.n_features);
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
        valid[r] = f < f_hi && p < n && !seg_skips(sg, f);
        rows[r] = valid[r] ? (uint32_t)__ldcs(in + (size_t)f * sg.in_fstride + p) : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < R; ++r) {
        if (f_lo + r * per >= f_hi) break;
        const uint32_t f = f_lo + r * per + sub;
        const bool left = valid[r] && left_bit(sg.bits, rows[r] & sg.row_mask);
        const unsigned lm = __ballot_sync(FULL, left) & gmask;
        const uint32_t rl = __popc(lm & lt);
        const uint32_t dst = left ? rl : nl + (p - rl);
        if (valid[r] && dst < n)
          __stcs(out + (size_t)f * sg.out_fstride + dst, (IdxT)rows[r]);
      }
    } else if (n <= 32) {
      uint32_t rows[FEAT_BLOCK];
#pragma unroll
      for (uint32_t r = 0; r < FEAT_BLOCK; ++r) {
        const uint32_t f = f_lo + r;
        rows[r] = (f < f_hi && lane < n) ? (uint32_t)__ldcs(in + (size_t)f * sg.in_fstride + lane) : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < FEAT_BLOCK; ++r) {
        const uint32_t f = f_lo + r;
        if (f >= f_hi) break;
        if (seg_skips(sg, f)) continue;
        const bool valid = lane < n;
        const bool left = valid && left_bit(sg.bits, rows[r] & sg.row_mask);
        const unsigned lm = __ballot_sync(FULL, left);
        const uint32_t rl = __popc(lm & lt);
        const uint32_t dst = left ? rl : nl + (lane - rl);
        if (valid && dst < n) __stcs(out + (size_t)f * sg.out_fstride + dst, (IdxT)rows[r]);
      }
    } else {
      // blocks of PART_ROUNDS rounds held in registers; the left count of the
      // earlier blocks (run) carries over, so segments longer than one block
      // (up to the fit's small_rows) stay with one warp
      for (uint32_t f = f_lo; f < f_hi; ++f) {
        if (seg_skips(sg, f)) continue;
        const IdxT* fin = in + (size_t)f * sg.in_fstride;
        IdxT* fout = out + (size_t)f * sg.out_fstride;
        uint32_t run = 0;
        for (uint32_t b0 = 0; b0 < n; b0 += PART_PIECE) {
          const uint32_t rounds = min(ceil_div(n - b0, 32), PART_ROUNDS);
          uint32_t rows[PART_ROUNDS];
#pragma unroll
          for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
            const uint32_t p = b0 + r * 32 + lane;
            rows[r] = (r < rounds && p < n) ? (uint32_t)__ldcs(fin + p) : 0u;
          }
#pragma unroll
          for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
            if (r >= rounds) break;
            const uint32_t p = b0 + r * 32 + lane;
            const bool valid = p < n;
            const bool left = valid && left_bit(sg.bits, rows[r] & sg.row_mask);
            const unsigned lm = __ballot_sync(FULL, left);
            const uint32_t rl = run + __popc(lm & lt);
            const uint32_t dst = left ? rl : nl + (p - rl);
            if (valid && dst < n) __stcs(fout + dst, (IdxT)rows[r]);
            run += __popc(lm);
          }
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
// Global -> shared bulk copy; src 16-byte aligned, bytes a multiple of 16;
// pol is the L2 policy of the source lines.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
      : "memory");
}

// Persistent CTAs; each claims a whole (segment, feature) chain (k_plan lists
// the active ones) from a ticket counter and streams its tiles in order, so the running count of
// left rows (the chain's carry) stays in a register and no CTA ever waits
// for another.  Index tiles arrive by TMA bulk copies into a ring of
// RING buffers, RING-1 tiles ahead of the one being partitioned.  Copies
// are 16-byte aligned and rounded, so they read up to 15 bytes past a
// tile's last element (list buffers carry that padding).

template <typename IdxT, uint32_t TILE>
__device__ __forceinline__ void issue_tile(const IdxT* seg_in, uint32_t n, uint32_t j, unsigned char* buf,
                                           uint64_t* bar, uint32_t* off_out, uint64_t pol) {
  const uint32_t lo = j * TILE;
  const uint32_t cnt = min(TILE, n - lo);
  const uintptr_t a = reinterpret_cast<uintptr_t>(seg_in + lo);
  const uintptr_t a0 = a & ~uintptr_t(15);
  const uintptr_t e1 = (a + (uintptr_t)cnt * sizeof(IdxT) + 15) & ~uintptr_t(15);
  *off_out = (uint32_t)((a - a0) / sizeof(IdxT));
  mbar_expect_tx(bar, (uint32_t)(e1 - a0));
  bulk_g2s(buf, reinterpret_cast<const void*>(a0), (uint32_t)(e1 - a0), bar, pol);
}

template <typename IdxT, uint32_t ROUNDS>
constexpr uint32_t ring_buf_bytes() {
  return BIG_WARPS * 32 * ROUNDS * sizeof(IdxT) + 128;
}

// Where a chain's partition runs.  CtaEnv: a k_part_big CTA of BIG_WARPS
// warps, mark bits read from global memory (L1).  GroupEnv: one group of
// BIG_WARPS warps of a k_part_seg CTA, mark bits staged in shared memory.
struct CtaEnv {
  const uint32_t* bits;
  __device__ uint32_t warp() const { return threadIdx.x >> 5; }
  __device__ bool leader() const { return threadIdx.x == 0; }
  __device__ void sync() const { __syncthreads(); }
  __device__ bool all(bool ok) const { return __syncthreads_and(ok); }
  __device__ bool left(uint32_t row) const { return left_bit(bits, row); }
};

constexpr uint32_t SEG_GROUPS = 4;  // k_part_seg: groups of BIG_WARPS warps per CTA
constexpr uint32_t SEG_THREADS = SEG_GROUPS * BIG_THREADS;

struct GroupEnv {
  const uint32_t* sbits;
  uint32_t g;
  __device__ uint32_t warp() const { return (threadIdx.x >> 5) - g * BIG_WARPS; }
  __device__ bool leader() const { return threadIdx.x == g * BIG_THREADS; }
  __device__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(BIG_THREADS) : "memory"); }
  __device__ bool all(bool ok) const {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(g + 1), "r"(BIG_THREADS)
        : "memory");
    return r != 0;
  }
  __device__ bool left(uint32_t row) const { return (sbits[row >> 5] >> (row & 31)) & 1u; }
};

// One tile of a chain: the left flags of the group's BIG_WARPS * 32 * ROUNDS
// positions, the group's prefix of left counts, and the stable stores;
// returns the tile's left count.  WHOLE: the tile is full, so positions need
// no range check.
template <typename IdxT, uint32_t ROUNDS, bool WHOLE, typename Env>
__device__ __forceinline__ uint32_t part_tile(const Env& env, const IdxT* rows, uint32_t cnt, uint32_t lo,
                                              const PartSeg& sg, uint32_t row_mask, IdxT* out, uint32_t n,
                                              uint32_t carry, uint32_t* s_wcnt) {
  const uint32_t lane = lane_id(), warp = env.warp();
  const unsigned lt = lanemask_lt();
  const uint32_t wlo = warp * (32 * ROUNDS);
  unsigned lmask[ROUNDS];
  IdxT e[ROUNDS];
  uint32_t wc = 0;
#pragma unroll
  for (uint32_t r = 0; r < ROUNDS; ++r) {
    const uint32_t q = wlo + r * 32 + lane;
    const bool in = WHOLE || q < cnt;
    e[r] = rows[in ? q : 0];
    const bool left = in && env.left((uint32_t)e[r] & row_mask);
    lmask[r] = __ballot_sync(FULL, left);
    wc += __popc(lmask[r]);
  }
  if (lane == 0) s_wcnt[warp] = wc;
  env.sync();
  // the warps' left counts: lane k of every warp holds warp k's, scanned over 8 lanes
  static_assert(BIG_WARPS == 8, "the count prefix scans 8 lanes");
  uint32_t v = s_wcnt[lane & 7u];
#pragma unroll
  for (uint32_t d = 1; d < 8; d <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL, v, d, 8);
    if ((lane & 7u) >= d) v += o;
  }
  const uint32_t total = __shfl_sync(FULL, v, 7);
  const uint32_t woff = warp ? __shfl_sync(FULL, v, warp - 1) : 0u;
  uint32_t run = carry + woff;
#pragma unroll
  for (uint32_t r = 0; r < ROUNDS; ++r) {
    const uint32_t q = wlo + r * 32 + lane;
    const bool left = (lmask[r] >> lane) & 1u;
    const uint32_t rl = run + __popc(lmask[r] & lt);
    if (WHOLE || q < cnt) {
      const uint32_t dst = left ? rl : sg.nl + (lo + q - rl);
      if (dst < n) __stcs(out + dst, e[r]);
    }
    run += __popc(lmask[r]);
  }
  return total;
}

// One (segment, feature) chain through a ring of RING tile buffers: tiles
// arrive by bulk copies RING-1 ahead of the one being partitioned; the left
// count carried between tiles is a register.  g counts the tiles this ring
// has consumed, uses[b] the completed phases of buffer b.  Returns false
// (error word set, the ring drained, bounded) when a copy did not arrive.
template <typename IdxT, uint32_t ROUNDS, uint32_t RING, typename Env>
__device__ __forceinline__ bool run_chain(const Env& env, const PartWork& w, const PartSeg& sg, uint32_t f,
                                          unsigned char* ring, uint64_t* bars, uint32_t* s_off, uint32_t* s_wcnt,
                                          uint32_t (&uses)[RING], uint32_t& g, uint64_t stream_pol) {
  constexpr uint32_t TILE = BIG_WARPS * 32 * ROUNDS;
  constexpr uint32_t BUF = ring_buf_bytes<IdxT, ROUNDS>();
  unsigned char(*sbuf)[BUF] = reinterpret_cast<unsigned char(*)[BUF]>(ring);
  const IdxT* in = reinterpret_cast<const IdxT*>(sg.in) + (size_t)f * sg.in_fstride;
  IdxT* out = reinterpret_cast<IdxT*>(sg.out) + (size_t)f * sg.out_fstride;
  const uint32_t n = sg.n;
  const uint32_t ntiles = ceil_div(n, TILE);
  if (env.leader())
    for (uint32_t j = 0; j < RING - 1 && j < ntiles; ++j)
      issue_tile<IdxT, TILE>(in, n, j, sbuf[(g + j) % RING], &bars[(g + j) % RING], &s_off[(g + j) % RING],
                             stream_pol);
  uint32_t carry = 0;
  for (uint32_t j = 0; j < ntiles; ++j, ++g) {
    const uint32_t b = g % RING;
    if (env.leader() && j + RING - 1 < ntiles) {  // refill the buffer freed by tile j-1
      const uint32_t bn = (g + RING - 1) % RING;
      issue_tile<IdxT, TILE>(in, n, j + RING - 1, sbuf[bn], &bars[bn], &s_off[bn], stream_pol);
    }
    bool ok = true;
    {
      uint32_t spins = 0;
      while (!mbar_try_wait(&bars[b], uses[b] & 1u)) {
        if (++spins > (SPIN_LIMIT << 2)) {
          ok = false;
          break;
        }
      }
    }
    if (!env.all(ok)) {
      // never read a tile that did not arrive: flag, drain the ring (bounded), leave
      if (env.leader()) atomicOr(w.error, DEV_ERR_TIMEOUT);
      for (uint32_t k = 0; k < RING && j + k < ntiles; ++k) {  // tiles j .. j+RING-1 may be in flight
        const uint32_t bb = (g + k) % RING;
        uint32_t spins = 0;
        while (!mbar_try_wait(&bars[bb], uses[bb] & 1u) && ++spins < (SPIN_LIMIT << 4)) {
        }
        uses[bb] += 1;
      }
      return false;
    }
    uses[b] += 1;
    const uint32_t lo = j * TILE;
    const uint32_t cnt = min(TILE, n - lo);
    const IdxT* rows = reinterpret_cast<const IdxT*>(sbuf[b]) + s_off[b];
    carry += cnt == TILE ? part_tile<IdxT, ROUNDS, true>(env, rows, cnt, lo, sg, sg.row_mask, out, n, carry, s_wcnt)
                         : part_tile<IdxT, ROUNDS, false>(env, rows, cnt, lo, sg, sg.row_mask, out, n, carry, s_wcnt);
    env.sync();  // tile buffer and s_wcnt free for reuse
  }
  return true;
}

template <typename IdxT, uint32_t ROUNDS, uint32_t RING, uint32_t MINB>
__global__ void __launch_bounds__(BIG_THREADS, MINB) k_part_big(PartWork w) {
  extern __shared__ __align__(128) unsigned char ring_smem[];
  __shared__ alignas(8) uint64_t bars[RING];
  __shared__ uint32_t s_off[RING];
  __shared__ uint32_t s_chain;
  __shared__ uint32_t s_wcnt[BIG_WARPS];
  const uint32_t chains = live(w, w.n_bchains, w.cap_bchains);
  const uint64_t stream_pol = l2_evict_first();  // list tiles are read once
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < RING; ++i) mbar_init(&bars[i], 1);
    mbar_fence_init();
  }
  uint32_t uses[RING];  // completed phases per ring buffer (uniform)
#pragma unroll
  for (uint32_t i = 0; i < RING; ++i) uses[i] = 0;
  uint32_t g = 0;  // tiles consumed by this CTA (ring position)
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_chain = atomicAdd(w.ticket, 1u);
    __syncthreads();
    const uint32_t c = s_chain;
    if (c >= chains) break;
    // a segment's chains are listed together: the chains in flight share few
    // segments (trees), so the mark bits they gather stay hot in L2
    const uint2 ch = w.bchains[c];
    const uint32_t f = ch.y;
    const PartSeg sg = w.big[ch.x];
    const CtaEnv env{sg.bits};
    if (!run_chain<IdxT, ROUNDS, RING>(env, w, sg, f, ring_smem, bars, s_off, s_wcnt, uses, g, stream_pol)) return;
  }
}

// Segments of at least HUGE_SEG rows, when the tree's mark bits fit shared
// memory (huge_partition_ok): one CTA of SEG_GROUPS groups per SM.  A work
// unit is a quad of the segment's active chains (k_plan lists them, padded
// to quads, so a quad never spans two segments); the CTA stages the
// segment's tree's mark bits in shared memory by one bulk copy (kept while
// consecutive units share the tree) and each group partitions one chain of
// the quad with a bit lookup in shared memory: a divergent load of 32 rows
// there costs a few bank cycles, against up to 32 L1 wavefronts.
template <typename IdxT, uint32_t ROUNDS, uint32_t RING>
__global__ void __launch_bounds__(SEG_THREADS, 1) k_part_seg(PartWork w) {
  constexpr uint32_t BUF = ring_buf_bytes<IdxT, ROUNDS>();
  extern __shared__ __align__(128) unsigned char seg_smem[];
  __shared__ alignas(8) uint64_t bars[SEG_GROUPS][RING];
  __shared__ alignas(8) uint64_t bits_bar;
  __shared__ uint32_t s_off[SEG_GROUPS][RING];
  __shared__ uint32_t s_wcnt[SEG_GROUPS][BIG_WARPS];
  __shared__ uint32_t s_unit;
  __shared__ uint32_t s_fail;
  const uint32_t bit_bytes = w.bit_words * 4u;
  uint32_t* sbits = reinterpret_cast<uint32_t*>(seg_smem);
  const uint32_t g = threadIdx.x / BIG_THREADS;
  unsigned char* ring = seg_smem + ((bit_bytes + 127u) & ~127u) + (size_t)g * RING * BUF;
  const uint32_t nq = live(w, w.n_hchains, w.cap_hchains) / SEG_GROUPS;
  const uint64_t stream_pol = l2_evict_first();
  const uint64_t keep_pol = l2_evict_last();  // mark bits are staged again by later units
  if (threadIdx.x == 0) {
    for (uint32_t k = 0; k < SEG_GROUPS; ++k)
      for (uint32_t i = 0; i < RING; ++i) mbar_init(&bars[k][i], 1);
    mbar_init(&bits_bar, 1);
    mbar_fence_init();
    s_fail = 0;
  }
  uint32_t uses[RING];
#pragma unroll
  for (uint32_t i = 0; i < RING; ++i) uses[i] = 0;
  uint32_t gpos = 0, bits_uses = 0;
  const uint32_t* staged = nullptr;
  while (true) {
    __syncthreads();  // every group is done with the previous unit (its bits, its chain)
    if (threadIdx.x == 0) s_unit = atomicAdd(w.ticket_huge, 1u);
    __syncthreads();
    const uint32_t u = s_unit;
    if (u >= nq || s_fail) break;
    const uint2 ch = w.hchains[u * SEG_GROUPS + g];
    const uint2 first = w.hchains[u * SEG_GROUPS];
    const PartSeg sg = w.huge[first.x];
    if (sg.bits != staged) {
      if (threadIdx.x == 0) {
        mbar_expect_tx(&bits_bar, bit_bytes);
        bulk_g2s(sbits, sg.bits, bit_bytes, &bits_bar, keep_pol);
      }
      uint32_t spins = 0;
      bool ok = true;
      while (!mbar_try_wait(&bits_bar, bits_uses & 1u)) {
        if (++spins > (SPIN_LIMIT << 2)) {
          ok = false;
          break;
        }
      }
      if (!__syncthreads_and(ok)) {  // drain the copy (bounded) and leave
        if (threadIdx.x == 0) atomicOr(w.error, DEV_ERR_TIMEOUT);
        spins = 0;
        while (!mbar_try_wait(&bits_bar, bits_uses & 1u) && ++spins < (SPIN_LIMIT << 4)) {
        }
        return;
      }
      bits_uses += 1;
      staged = sg.bits;
    }
    if (ch.y != NONE) {
      const GroupEnv env{sbits, g};
      if (!run_chain<IdxT, ROUNDS, RING>(env, w, w.huge[ch.x], ch.y, ring, bars[g], s_off[g], s_wcnt[g], uses, gpos,
                                         stream_pol))
        s_fail = 1;
    }
  }
}

template <typename K>
int resident_blocks(K kernel, int threads, size_t dyn_smem = 0) {
  static const int sms = [] {  // initialized once, thread-safe
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, dyn_smem);
  return sms * (per > 0 ? per : 1);
}

template <typename IdxT, uint32_t ROUNDS, uint32_t RING, uint32_t MINB>
int launch_big_v(const PartWork& w, uint64_t want, cudaStream_t st) {
  const size_t smem = RING * ring_buf_bytes<IdxT, ROUNDS>();
  // per instantiation (the attribute is per device function); once, thread-safe
  static const cudaError_t configured = cudaFuncSetAttribute(
      k_part_big<IdxT, ROUNDS, RING, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  CT_CUDA_TRY(configured);
  const int cap = resident_blocks(k_part_big<IdxT, ROUNDS, RING, MINB>, BIG_THREADS, smem);
  k_part_big<IdxT, ROUNDS, RING, MINB><<<(uint32_t)std::min<uint64_t>(want, cap), BIG_THREADS, smem, st>>>(w);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

// The shapes of CT_PART_*: tile (8 warps x ROUNDS rounds of 32), ring
// buffers, CTAs per SM.  The default, 2,048-element tiles in two buffers at
// six CTAs per SM (at most 40 registers), leaves most of the SM's L1 to the
// mark bits the chains gather; the others trade tile length, copies in
// flight and occupancy, for the autotuner to time.
template <typename IdxT>
int launch_big(const PartWork& w, uint64_t want, cudaStream_t st) {
  switch (w.shape) {
    case CT_PART_1024_R3_B8: return launch_big_v<IdxT, 4, 3, 8>(w, want, st);
    case CT_PART_4096_R2_B4: return launch_big_v<IdxT, 16, 2, 4>(w, want, st);
    case CT_PART_2048_R3_B4: return launch_big_v<IdxT, 8, 3, 4>(w, want, st);
    default: return launch_big_v<IdxT, 8, 2, 6>(w, want, st);
  }
}

}  // namespace

template <typename IdxT>
int launch_seg(const PartWork& w, cudaStream_t st) {
  constexpr uint32_t ROUNDS = 8, RING = 2;
  const size_t smem = (((size_t)w.bit_words * 4 + 127) & ~size_t(127)) +
                      (size_t)SEG_GROUPS * RING * ring_buf_bytes<IdxT, ROUNDS>();
  // per instantiation, the largest staging it can take; once, thread-safe
  static const cudaError_t configured = cudaFuncSetAttribute(
      k_part_seg<IdxT, ROUNDS, RING>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)((size_t)HUGE_BITS_MAX + 128 + (size_t)SEG_GROUPS * RING * ring_buf_bytes<IdxT, ROUNDS>()));
  CT_CUDA_TRY(configured);
  int dev = 0, sms = 0;
  CT_CUDA_TRY(cudaGetDevice(&dev));
  CT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  k_part_seg<IdxT, ROUNDS, RING><<<(uint32_t)std::max(1, sms), SEG_THREADS, smem, st>>>(w);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int launch_seg_partition(uint32_t index_bytes, const PartWork& w, uint64_t bound_small, uint64_t bound_tiles,
                         cudaStream_t st) {
  if (bound_tiles > 0 && w.huge && huge_partition_ok(w.bit_words)) {
    if (index_bytes == 2) CT_TRY(launch_seg<uint16_t>(w, st));
    else CT_TRY(launch_seg<uint32_t>(w, st));
  }
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
    const uint64_t want = bound_tiles * w.n_features;  // >= number of (big segment, feature) chains
    if (index_bytes == 2) CT_TRY(launch_big<uint16_t>(w, want, st));
    else CT_TRY(launch_big<uint32_t>(w, want, st));
  }
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

}  // namespace ct
