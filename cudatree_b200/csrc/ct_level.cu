// Level-step kernels of the split search and the stable partition.
//
//   k_select       feature subset of each node (reference DFS: first m of a
//                  shuffled permutation, random_tree.py:624; BFS: non-constant
//                  features only, bfs_module.cu:130-140)
//   k_scan_hist    class histograms of all but the last piece of long segments
//   k_scan_carry   exclusive per-class prefix over those pieces
//                  (reference scan_gini_large + scan_reduce, dfs_module.cu:24-106)
//   k_split_scan   Gini scan of one piece: per-element class rank via
//                  __match_any_sync, int64 warp scans of the sum of squared
//                  counts, fp64 impurity (reference compute_2d, dfs_module.cu:310-443)
//   k_scan_two_valued  the same result for pieces of two-valued features:
//                  a search for the node's value boundary instead of a scan
//   k_split_reduce min-impurity reduction + threshold
//                  (reference reduce_2d / find_min_imp / get_thresholds)
//   k_plan         node record, child ids, partition work list
//   k_fill_mark    mark bits + left class totals (reference fill_table)
//   (partition)    stable partition of every feature's node range: plan and
//                  mark table here, the kernels in ct_partition.cu
//                  (reference scan_reshuffle, dfs_module.cu:224-307)
//   k_children     child records for the next step
#include <algorithm>
#include <cfloat>

#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr uint32_t SCAN_BATCH = 4;  // rounds of 32 whose loads are issued together

__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000ll); }

__device__ __forceinline__ uint32_t global_warp() {
  return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ uint32_t total_warps() { return (gridDim.x * blockDim.x) >> 5; }

// Items of a warp-per-item launch.  A warp takes item global_warp() first;
// when the grid does not cover every item (a persistent launch), it then
// claims the items past the grid in order from a counter, so uneven items
// balance as they do with one warp per item.  Warp-collective.
template <typename F>
__device__ __forceinline__ void for_items(uint32_t count, uint32_t* claim, F item) {
  const uint32_t nw = total_warps();
  uint32_t w = global_warp();
  while (w < count) {
    item(w);
    __syncwarp();
    if (nw >= count) break;
    uint32_t k = 0;
    if (lane_id() == 0) k = atomicAdd(claim, 1u);
    w = nw + __shfl_sync(FULL, k, 0);
  }
}

__device__ __forceinline__ uint32_t read_error(const Counters* c) {
  return *reinterpret_cast<const volatile uint32_t*>(&c->error);
}
// Work-list count clamped to its capacity; 0 once an earlier kernel of the
// step flagged an error, so no kernel reads a record that was not written.
__device__ __forceinline__ uint32_t live_count(const LevelScratch& s, uint32_t count, uint32_t cap) {
  return read_error(s.ctr) ? 0u : min(count, cap);
}

// (score, pos) lexicographic minimum across the warp.
__device__ __forceinline__ void warp_argmin2(double& score, uint32_t& pos, float& p, float& q) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    double os = __shfl_xor_sync(FULL, score, s);
    uint32_t op = __shfl_xor_sync(FULL, pos, s);
    float a = __shfl_xor_sync(FULL, p, s);
    float b = __shfl_xor_sync(FULL, q, s);
    if (os < score || (os == score && op < pos)) {
      score = os;
      pos = op;
      p = a;
      q = b;
    }
  }
}

// ------------------------------------------------------------------------
// Virtual features: per-node counts from the node's row list (list slot
// vslot: its rows in row order) and the rows' value bits (vrow).
//
//   k_vpieces    cuts each node's row list into pieces of VPIECE rows and
//                zeroes the node's counts
//   k_vcount     per piece: for every virtual feature f and class c, the rows
//                with f's high value and class c (one shared-memory add per
//                set value bit: one-hot rows have one per group), added into
//                vcls[node][f][c], and their sum into vcnt[node][f].
//                k_select takes a virtual feature as non-constant in a node
//                when 0 < vcnt < n; k_split_reduce scores its one candidate
//                (the last low-value row) from vcls.
__device__ __forceinline__ void vpieces_item(const View& v, const StepLists& lists, const LevelScratch& s,
                                             uint32_t w) {
  const uint32_t lane = lane_id();
  const ct_node nd = lists.nodes[w];
  const uint32_t fc = v.n_features * v.n_classes;
  for (uint32_t f = lane; f < 64; f += 32) s.vcnt[(size_t)w * 64 + f] = 0;
  for (uint32_t i = lane; i < fc; i += 32) s.vcls[(size_t)w * fc + i] = 0;
  if (nd.n < 2) return;
  const uint32_t np = ceil_div(nd.n, VPIECE);
  uint32_t base = 0;
  if (lane == 0) {
    base = atomicAdd(&s.ctr->n_vpieces, np);
    if (base + (uint64_t)np > s.cap_vpieces) {
      atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
      base = NONE;
    }
  }
  base = __shfl_sync(FULL, base, 0);
  if (base == NONE) return;
  for (uint32_t j = lane; j < np; j += 32) s.vpieces[base + j] = make_uint2(w, j);
}

__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_vpieces(View v, LevelScratch s) {
  const uint32_t count = min(s.ctr->n_nodes, s.cap_nodes);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_VPIECES], [&](uint32_t w) { vpieces_item(v, sl, s, w); });
}

// Per-warp shared memory: [n_features][n_classes] counts.
template <typename IdxT, typename LabT>
__device__ __forceinline__ void vcount_item(const View& v, const StepLists& lists, const LevelScratch& s,
                                            uint32_t* cnt, uint32_t pi) {
  const uint32_t lane = lane_id();
  const uint32_t C = v.n_classes, fc = v.n_features * C;
  const uint2 pc = s.vpieces[pi];
  const ct_node nd = lists.nodes[pc.x];
  const IdxT* rl = list_ptr<IdxT>(v, nd.buf, nd.slot, v.vslot) + nd.start;
  const uint32_t lo = pc.y * VPIECE;
  const uint32_t hi = min(lo + VPIECE, nd.n);
  for (uint32_t i = lane; i < fc; i += 32) cnt[i] = 0;
  __syncwarp();
  // VB rows per lane: their entry loads, then their value-bit gathers, are in
  // flight together (one row at a time left the loop waiting on two loads)
  constexpr uint32_t VB = 8;
  for (uint32_t i0 = lo; i0 < hi; i0 += 32 * VB) {
    uint32_t e[VB];
    uint64_t bits[VB];
#pragma unroll
    for (uint32_t r = 0; r < VB; ++r) {
      const uint32_t i = i0 + r * 32 + lane;
      e[r] = i < hi ? (uint32_t)__ldcs(rl + i) : 0u;
    }
#pragma unroll
    for (uint32_t r = 0; r < VB; ++r)
      bits[r] = i0 + r * 32 + lane < hi ? __ldg(v.vrow + entry_row(v, e[r])) : 0ull;
#pragma unroll
    for (uint32_t r = 0; r < VB; ++r) {
      if (!bits[r]) continue;
      const uint32_t lab = entry_label<LabT>(v, e[r]);
      for (uint64_t b = bits[r]; b; b &= b - 1)
        atomicAdd(&cnt[((uint32_t)__ffsll((long long)b) - 1) * C + lab], 1u);
    }
  }
  __syncwarp();
  if (lane == 0) atomicAdd(&s.ctr->vrows, (unsigned long long)(hi - lo));
  uint32_t* out = s.vcls + (size_t)pc.x * fc;
  for (uint32_t i = lane; i < fc; i += 32)
    if (cnt[i]) atomicAdd(&out[i], cnt[i]);
  for (uint32_t f = lane; f < v.n_features; f += 32) {
    if (!is_virtual(v, f)) continue;
    uint32_t t = 0;
    for (uint32_t c = 0; c < C; ++c) t += cnt[f * C + c];
    if (t) atomicAdd(&s.vcnt[(size_t)pc.x * 64 + f], t);
  }
}

template <typename IdxT, typename LabT>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_vcount(View v, LevelScratch s) {
  extern __shared__ uint32_t smem[];
  uint32_t* cnt = smem + (threadIdx.x >> 5) * v.n_features * v.n_classes;
  const uint32_t count = live_count(s, s.ctr->n_vpieces, s.cap_vpieces);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_VCOUNT], [&](uint32_t pi) { vcount_item<IdxT, LabT>(v, sl, s, cnt, pi); });
}

// ------------------------------------------------------------------------
template <typename IdxT, bool Q>
__device__ __forceinline__ void select_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                            uint32_t scan_piece, uint32_t w) {
  const uint32_t lane = lane_id();
  const ct_node nd = lists.nodes[w];
  CT_JOB_VIEW(v, vb, nd.slot);
  const uint32_t m = v.max_features;
  // constant features (lists not current)
  const uint64_t* cmask = lists.node_mask ? lists.node_mask + (size_t)w * v.mask_stride : nullptr;
  uint32_t taken = 0;
  uint64_t vsel = 0;  // selected slots that hold virtual features (m <= 64 when there are any)
  if (nd.n >= 2) {
    for (uint32_t i0 = 0; i0 < v.n_features && taken < m; i0 += 32) {
      const uint32_t i = i0 + lane;
      bool usable = false, virt = false;
      uint32_t f = 0;
      if (i < v.n_features) {
        f = feature_perm(i, v.n_features, nd.key, v.feistel_h);
        virt = is_virtual(v, f);
        if (virt) {  // non-constant: some but not all rows take the high value
          const uint32_t nb = s.vcnt[(size_t)w * 64 + f];
          usable = nb > 0 && nb < nd.n;
        } else if (!mask_bit(cmask, f)) {
          const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, f) + nd.start;
          const float* xf = v.x_fm + (size_t)f * v.n_rows;
          usable = xf[entry_row(v, lst[0])] != xf[entry_row(v, lst[nd.n - 1])];
        }
      }
      const unsigned mask = __ballot_sync(FULL, usable);
      const uint32_t rank = __popc(mask & lanemask_lt());
      const bool keep = usable && taken + rank < m;
      if (keep) s.sel[(size_t)w * v.sel_stride + taken + rank] = f;
      const uint64_t vb = (keep && virt) ? 1ull << (taken + rank) : 0ull;
      vsel |= ((uint64_t)__reduce_or_sync(FULL, (uint32_t)(vb >> 32)) << 32) | __reduce_or_sync(FULL, (uint32_t)vb);
      taken += min((uint32_t)__popc(mask), m - taken);
    }
  }
  // scan pieces for the materialized slots only (virtual ones are scored from counts)
  const uint32_t tmat = taken - (uint32_t)__popcll(vsel);
  const uint32_t pps = ceil_div(nd.n, scan_piece);
  uint32_t npieces = tmat * pps;
  uint32_t base = 0, cbase = 0;
  if (lane == 0) {
    if (tmat) atomicAdd(&s.ctr->scan_elems, (unsigned long long)tmat * nd.n);
    if (npieces) base = atomicAdd(&s.ctr->n_scan_pieces, npieces);
    if (npieces && pps > 1) cbase = atomicAdd(&s.ctr->n_carry, npieces);
    const bool overflow = (base + (uint64_t)npieces > s.cap_scan) ||
                          (pps > 1 && cbase + (uint64_t)npieces > s.cap_carry);
    if (overflow) {
      atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
      npieces = 0;
    }
    s.nsel[w] = taken;
    s.piece_base[w] = base;
    s.piece_cnt[w] = npieces;
  }
  npieces = __shfl_sync(FULL, npieces, 0);
  base = __shfl_sync(FULL, base, 0);
  cbase = __shfl_sync(FULL, cbase, 0);
  __syncwarp();  // the slots' features in s.sel, written by other lanes
  // Besides the piece records, the piece of every carry row (k_scan_hist and
  // k_scan_carry walk only the pieces of multi-piece segments) and the list
  // of two-valued features' pieces (k_scan_two_valued walks only those), so
  // that those kernels claim no item they have nothing to do for.
  for (uint32_t q0 = 0; q0 < npieces; q0 += 32) {
    const uint32_t q = q0 + lane;
    bool tv = false;
    if (q < npieces) {
      ScanPiece pc;
      pc.node = w;
      const uint32_t k = q / pps;  // k-th materialized slot
      pc.slot = k;
      if (vsel) {
        uint32_t slot = 0;
        for (uint32_t left = k;; ++slot)
          if (!((vsel >> slot) & 1ull) && left-- == 0) break;
        pc.slot = slot;
      }
      pc.j = q - k * pps;
      pc.npieces = pps;
      pc.carry = cbase + q;
      pc.pad[0] = pc.pad[1] = pc.pad[2] = 0;
      s.pieces[base + q] = pc;
      if (pps > 1) s.carry_piece[cbase + q] = base + q;
      tv = two_valued(v, s.sel[(size_t)w * v.sel_stride + pc.slot]);
    }
    const unsigned tm = __ballot_sync(FULL, tv);
    if (tm) {  // n_tv <= n_scan_pieces <= cap_scan
      uint32_t tb = 0;
      if (lane == 0) tb = atomicAdd(&s.ctr->n_tv, (uint32_t)__popc(tm));
      tb = __shfl_sync(FULL, tb, 0);
      if (tv) s.tv_pieces[tb + __popc(tm & lanemask_lt())] = base + q;
    }
  }
}

template <typename IdxT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_select(View v, LevelScratch s) {
  const uint32_t count = min(s.ctr->n_nodes, s.cap_nodes);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_SELECT], [&](uint32_t w) { select_item<IdxT, Q>(v, sl, s, sl.scan_piece, w); });
}

// ------------------------------------------------------------------------
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void scan_hist_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                               uint32_t scan_piece, uint32_t* cnt, uint32_t pi) {
  const uint32_t C = vb.n_classes;
  const uint32_t lane = lane_id();
  const ScanPiece pc = s.pieces[pi];
  if (pc.npieces <= 1 || pc.j + 1 == pc.npieces) return;
  const ct_node nd = lists.nodes[pc.node];
  CT_JOB_VIEW(v, vb, nd.slot);
  const uint32_t f = s.sel[(size_t)pc.node * v.sel_stride + pc.slot];
  const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, f) + nd.start;
  const uint32_t lo = pc.j * scan_piece;
  const uint32_t hi = min(lo + scan_piece, nd.n);
  if (C <= 8 && scan_piece <= 32 * 255) {
    // each lane counts its (at most 255) positions in 8-bit fields of one
    // register, one field per class; one warp sum per class at the end
    uint64_t pk = 0;
    for (uint32_t base = lo; base < hi; base += 32 * SCAN_BATCH) {
      uint32_t rows[SCAN_BATCH];
#pragma unroll
      for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
        const uint32_t p = base + r * 32 + lane;
        rows[r] = p < hi ? (uint32_t)__ldcs(lst + p) : 0u;
      }
#pragma unroll
      for (uint32_t r = 0; r < SCAN_BATCH; ++r)
        if (base + r * 32 + lane < hi) pk += 1ull << (8 * entry_label<LabT>(v, rows[r]));
    }
    uint32_t* out = s.carry + (size_t)pc.carry * C;
    for (uint32_t c = 0; c < C; ++c) {
      const uint32_t t = warp_sum_u32((uint32_t)(pk >> (8 * c)) & 0xffu);
      if (lane == 0) out[c] = t;
    }
    return;
  }
  for (uint32_t c = lane; c < C; c += 32) cnt[c] = 0;
  __syncwarp();
  for (uint32_t base = lo; base < hi; base += 32 * SCAN_BATCH) {
    uint32_t rows[SCAN_BATCH], cs[SCAN_BATCH];
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const uint32_t p = base + r * 32 + lane;
      rows[r] = p < hi ? (uint32_t)__ldcs(lst + p) : 0u;
    }
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r)
      cs[r] = (base + r * 32 + lane < hi) ? entry_label<LabT>(v, rows[r]) : NONE;
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const unsigned grp = __match_any_sync(FULL, cs[r]);
      if (cs[r] != NONE && (grp >> lane) == 1u) cnt[cs[r]] += __popc(grp);
      __syncwarp();
    }
  }
  uint32_t* out = s.carry + (size_t)pc.carry * C;
  for (uint32_t c = lane; c < C; c += 32) out[c] = cnt[c];
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_scan_hist(View v, LevelScratch s) {
  extern __shared__ uint32_t smem[];
  uint32_t* cnt = smem + (threadIdx.x >> 5) * v.n_classes;
  const uint32_t count = live_count(s, s.ctr->n_carry, s.cap_carry);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_HIST],
            [&](uint32_t i) { scan_hist_item<IdxT, LabT, Q>(v, sl, s, sl.scan_piece, cnt, s.carry_piece[i]); });
}

__device__ __forceinline__ void scan_carry_item(const LevelScratch& s, uint32_t C, uint32_t pi) {
  const uint32_t lane = lane_id();
  const ScanPiece pc = s.pieces[pi];
  if (pc.npieces <= 1 || pc.j != 0) return;
  // per class, an exclusive prefix over the segment's pieces, 32 pieces per round
  for (uint32_t c = 0; c < C; ++c) {
    uint32_t run = 0;
    for (uint32_t j0 = 0; j0 < pc.npieces; j0 += 32) {
      const uint32_t j = j0 + lane;
      uint32_t* h = s.carry + (size_t)(pc.carry + j) * C + c;
      const uint32_t t = (j + 1 < pc.npieces) ? *h : 0u;
      const uint32_t incl = (uint32_t)warp_incl_scan_i32((int32_t)t);
      if (j < pc.npieces) *h = run + incl - t;
      run += __shfl_sync(FULL, incl, 31);
    }
  }
}

__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_scan_carry(LevelScratch s, uint32_t C) {
  const uint32_t count = live_count(s, s.ctr->n_carry, s.cap_carry);
  for_items(count, &s.ctr->claim[ITEM_CARRY], [&](uint32_t i) { scan_carry_item(s, C, s.carry_piece[i]); });
}

// ------------------------------------------------------------------------
// Split scan of one piece of a two-valued feature.  In a node's sorted list
// such a feature is a run of its low value a followed by a run of its high
// value b, so the only candidate position is the last a (when a + 1e-5 < b:
// is_candidate, dfs_module.cu:400), and the left class counts there are the
// piece's carry plus the classes of the piece's entries up to it.  The piece
// holding that position (x[lo] == a and x[hi] == b, or hi == n) finds it with
// a 32-way search over x and scores it with the scan's exact arithmetic; the
// other pieces report no candidate.  Same result as the general scan, with
// a few gathers per piece instead of one per position.
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void two_valued_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                                uint32_t scan_piece, uint32_t* cnt, uint32_t pi) {
  const uint32_t C = vb.n_classes;
  const uint32_t* tot = lists.tot;
  const uint32_t lane = lane_id();
  const ScanPiece pc = s.pieces[pi];
  const ct_node nd = lists.nodes[pc.node];
  CT_JOB_VIEW(v, vb, nd.slot);
  const uint32_t f = s.sel[(size_t)pc.node * v.sel_stride + pc.slot];
  if (!two_valued(v, f)) return;  // k_split_scan's piece
  const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, f) + nd.start;
  const float* xf = v.x_fm + (size_t)f * v.n_rows;
  const uint32_t* carry = pc.npieces > 1 ? s.carry + (size_t)pc.carry * C : nullptr;
  PieceBest* out = s.best + pi;
  const uint32_t n = nd.n;
  const uint32_t lo = pc.j * scan_piece;
  const uint32_t hi = min(lo + scan_piece, n);
  const float a = xf[entry_row(v, lst[0])];
  const float b = xf[entry_row(v, lst[n - 1])];
  PieceBest pb;
  pb.score = dinf();
  pb.pos = NONE;
  pb.il = 0.f;
  pb.ir = 0.f;
  pb.pad = 0;
  const bool owns = is_candidate_sorted(a, b) && xf[entry_row(v, lst[lo])] == a &&
                    (hi == n || xf[entry_row(v, lst[hi])] == b);
  if (owns) {
    // last position with x == a in [lo, e), e = min(hi, n - 1): x[L] == a and
    // x[R] == b throughout; 32 probes of the interior per round
    uint32_t L = lo, R = min(hi, n - 1);
    while (R - L > 1) {
      const uint32_t k = R - L - 1;
      const uint32_t q = L + 1 + (uint32_t)(((uint64_t)k * lane) / 32u);  // every interior position when k <= 32
      const unsigned m = __ballot_sync(FULL, xf[entry_row(v, lst[q])] == a);
      const uint32_t c = __popc(m);  // probes see a on lanes [0, c): the values are sorted
      const uint32_t ql = __shfl_sync(FULL, q, c > 0 ? c - 1 : 0);
      const uint32_t qr = __shfl_sync(FULL, q, c < 32 ? c : 31);
      if (c > 0) L = ql;
      if (c < 32) R = qr;
    }
    const uint32_t p = L;
    // classes of the entries [lo, p]
    const uint32_t cnt_n = p - lo + 1;
    for (uint32_t c = lane; c < C; c += 32) cnt[c] = 0;
    __syncwarp();
    if (C <= 8 && cnt_n <= 32 * 255) {
      uint64_t pk = 0;  // 8-bit field per class, at most 255 entries per lane
      for (uint32_t i = lo + lane; i <= p; i += 32) pk += 1ull << (8 * entry_label<LabT>(v, (uint32_t)__ldcs(lst + i)));
      for (uint32_t c = 0; c < C; ++c) {
        const uint32_t t = warp_sum_u32((uint32_t)(pk >> (8 * c)) & 0xffu);
        if (lane == 0) cnt[c] = t;
      }
    } else {
      for (uint32_t i0 = lo; i0 <= p; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t c = i <= p ? entry_label<LabT>(v, (uint32_t)__ldcs(lst + i)) : NONE;
        const unsigned grp = __match_any_sync(FULL, c);
        if (c != NONE && (grp >> lane) == 1u) cnt[c] += __popc(grp);
        __syncwarp();
      }
    }
    __syncwarp();
    int64_t sl = 0, sr = 0;
    for (uint32_t c = lane; c < C; c += 32) {
      const int64_t l = (int64_t)cnt[c] + (carry ? carry[c] : 0u);
      const int64_t r = (int64_t)tot[(size_t)pc.node * C + c] - l;
      sl += l * l;
      sr += r * r;
    }
    sl = warp_sum_i64(sl);
    sr = warp_sum_i64(sr);
    const double nn = (double)n;
    const double nl = (double)(p + 1);
    const double nr = __dsub_rn(nn, nl);
    const double gl = gini_part(sl, nl, nn);
    const double gr = gini_part(sr, nr, nn);
    pb.score = __dadd_rn(gl, gr);
    pb.pos = p;
    pb.il = __double2float_rn(gl);
    pb.ir = __double2float_rn(gr);
  }
  if (lane == 0) *out = pb;
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_scan_two_valued(View v, LevelScratch s) {
  extern __shared__ uint32_t smem[];
  uint32_t* cnt = smem + (threadIdx.x >> 5) * v.n_classes;
  const uint32_t count = live_count(s, s.ctr->n_tv, s.cap_scan);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_TWO_VALUED],
            [&](uint32_t i) { two_valued_item<IdxT, LabT, Q>(v, sl, s, sl.scan_piece, cnt, s.tv_pieces[i]); });
}

// ------------------------------------------------------------------------
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void split_scan_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                                uint32_t scan_piece, uint32_t* cnt, uint32_t pi) {
  const uint32_t C = vb.n_classes;
  const uint32_t* tot = lists.tot;
  uint32_t* T = cnt + C;
  const uint32_t lane = lane_id();
  const ScanPiece pc = s.pieces[pi];
  const ct_node nd = lists.nodes[pc.node];
  CT_JOB_VIEW(v, vb, nd.slot);
  const uint32_t f = s.sel[(size_t)pc.node * v.sel_stride + pc.slot];
  if (two_valued(v, f)) return;  // k_scan_two_valued's piece
  const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, f) + nd.start;
  const float* xf = v.x_fm + (size_t)f * v.n_rows;
  const uint32_t* carry = pc.npieces > 1 ? s.carry + (size_t)pc.carry * C : nullptr;
  int64_t sl = 0, sr = 0;
  for (uint32_t c = lane; c < C; c += 32) {
    const uint32_t k = carry ? carry[c] : 0u;
    const uint32_t t = tot[(size_t)pc.node * C + c];
    cnt[c] = k;
    T[c] = t;
    const int64_t r = (int64_t)t - (int64_t)k;
    sl += (int64_t)k * k;
    sr += r * r;
  }
  sl = warp_sum_i64(sl);
  sr = warp_sum_i64(sr);
  __syncwarp();
  const uint32_t n = nd.n;
  const bool narrow = n < (1u << 25);
  const double nn = (double)n;
  const uint32_t lo = pc.j * scan_piece;
  const uint32_t hi = min(lo + scan_piece, n);
  double best = dinf();
  uint32_t bpos = NONE;
  float bil = 0.f, bir = 0.f;
  const unsigned lt = lanemask_lt();
  // Software pipeline over batches of SCAN_BATCH rounds: while batch b is
  // scanned, the label/value gathers of batch b+1 and the index loads of
  // batch b+2 are in flight.
  constexpr uint32_t B = 32 * SCAN_BATCH;
  uint32_t rows_n[SCAN_BATCH], cs[SCAN_BATCH];
  float xs[SCAN_BATCH];
  const uint64_t keep = l2_evict_last();
  {
    uint32_t rows[SCAN_BATCH];
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const uint32_t p = lo + r * 32 + lane;
      rows[r] = p < hi ? (uint32_t)__ldcs(lst + p) : 0u;
      const uint32_t q = p + B;
      rows_n[r] = q < hi ? (uint32_t)__ldcs(lst + q) : 0u;
    }
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const bool valid = lo + r * 32 + lane < hi;
      cs[r] = valid ? entry_label<LabT>(v, rows[r]) : NONE;
      xs[r] = valid ? ld_keep(xf + entry_row(v, rows[r]), keep) : 0.f;
    }
  }
  for (uint32_t base = lo; base < hi; base += B) {
    uint32_t cs_n[SCAN_BATCH];
    float xs_n[SCAN_BATCH];
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const bool valid = base + B + r * 32 + lane < hi;
      cs_n[r] = valid ? entry_label<LabT>(v, rows_n[r]) : NONE;
      xs_n[r] = valid ? ld_keep(xf + entry_row(v, rows_n[r]), keep) : 0.f;
    }
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const uint32_t q = base + 2 * B + r * 32 + lane;
      rows_n[r] = q < hi ? (uint32_t)__ldcs(lst + q) : 0u;
    }
    const float x_e = __shfl_sync(FULL, xs_n[0], 0);  // first value of the next batch
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      const uint32_t p = base + r * 32 + lane;
      const bool valid = p < hi;
      const uint32_t c = cs[r];
      const float x = xs[r];
      float xn = __shfl_down_sync(FULL, x, 1);
      const float first_next = (r + 1 < SCAN_BATCH) ? __shfl_sync(FULL, xs[r + 1 < SCAN_BATCH ? r + 1 : r], 0) : x_e;
      if (lane == 31) xn = first_next;
      if (valid && p + 1 == hi && p + 1 < n) xn = xf[entry_row(v, lst[p + 1])];  // next piece's first element
      const unsigned grp = __match_any_sync(FULL, c);
      uint32_t k = 0;
      int64_t tc = 0;
      if (valid) {
        k = cnt[c] + __popc(grp & lt);
        tc = T[c];
      }
      __syncwarp();
      if (valid && (grp >> lane) == 1u) cnt[c] += __popc(grp);
      __syncwarp();
      const int64_t dl = valid ? 2 * (int64_t)k + 1 : 0;
      const int64_t dr = valid ? 1 - 2 * (tc - (int64_t)k) : 0;
      int64_t il, ir, tl, tr;  // inclusive warp prefix and warp total of each increment
      if (narrow) {  // |partial sums| <= 32 (2n + 1) < 2^31
        const int32_t a = warp_incl_scan_i32((int32_t)dl), b = warp_incl_scan_i32((int32_t)dr);
        il = a;
        ir = b;
        tl = __shfl_sync(FULL, a, 31);
        tr = __shfl_sync(FULL, b, 31);
      } else {
        il = warp_incl_scan_i64(dl);
        ir = warp_incl_scan_i64(dr);
        tl = __shfl_sync(FULL, il, 31);
        tr = __shfl_sync(FULL, ir, 31);
      }
      const int64_t SL = sl + il;
      const int64_t SR = sr + ir;
      sl += tl;
      sr += tr;
      if (valid && p + 1 < n && is_candidate_sorted(x, xn)) {
        const double nl = (double)(p + 1);
        const double nr = __dsub_rn(nn, nl);
        const double gl = gini_part(SL, nl, nn);
        const double gr = gini_part(SR, nr, nn);
        const double sc = __dadd_rn(gl, gr);
        if (sc < best) {
          best = sc;
          bpos = p;
          bil = __double2float_rn(gl);
          bir = __double2float_rn(gr);
        }
      }
    }
#pragma unroll
    for (uint32_t r = 0; r < SCAN_BATCH; ++r) {
      cs[r] = cs_n[r];
      xs[r] = xs_n[r];
    }
  }
  warp_argmin2(best, bpos, bil, bir);
  if (lane == 0) {
    PieceBest pb;
    pb.score = best;
    pb.pos = bpos;
    pb.il = bil;
    pb.ir = bir;
    pb.pad = 0;
    s.best[pi] = pb;
  }
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK, 7)  // 72 registers: 28 warps per SM hide more of the scan's latency
k_split_scan(View v, LevelScratch s) {
  extern __shared__ uint32_t smem[];
  uint32_t* cnt = smem + (threadIdx.x >> 5) * 2 * v.n_classes;
  const uint32_t count = live_count(s, s.ctr->n_scan_pieces, s.cap_scan);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_SCAN],
            [&](uint32_t pi) { split_scan_item<IdxT, LabT, Q>(v, sl, s, sl.scan_piece, cnt, pi); });
}

// ------------------------------------------------------------------------
template <typename IdxT, bool Q>
__device__ __forceinline__ void split_reduce_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                                  uint32_t w) {
  const uint32_t lane = lane_id();
  const uint32_t base = s.piece_base[w];
  const uint32_t cnt = s.piece_cnt[w];
  CT_JOB_VIEW(v, vb, Q ? lists.nodes[w].slot : 0u);
  const uint32_t m = v.sel_stride;
  double best = dinf();
  uint32_t bf = NONE, bp = NONE;
  float il = 0.f, ir = 0.f;
  for (uint32_t q = lane; q < cnt; q += 32) {
    const PieceBest pb = s.best[base + q];
    const uint32_t f = s.sel[(size_t)w * m + s.pieces[base + q].slot];
    if (pb.score < best || (pb.score == best && (f < bf || (f == bf && pb.pos < bp)))) {
      best = pb.score;
      bf = f;
      bp = pb.pos;
      il = pb.il;
      ir = pb.ir;
    }
  }
  warp_argmin3(best, bf, bp, il, ir);
  if (v.vmask) {
    // virtual features: one candidate each, the last low-value row, with the
    // class counts of the high-value rows from k_vcount (the same exact
    // arithmetic as the scan; the same (score, feature, position) order)
    const uint32_t nsel = s.nsel[w];
    const ct_node nd = lists.nodes[w];
    const uint32_t C = v.n_classes;
    const double nn = (double)nd.n;
    for (uint32_t q = 0; q < nsel; ++q) {
      const uint32_t f = s.sel[(size_t)w * m + q];
      if (!is_virtual(v, f)) continue;
      const float2 lh = v.vval[f];
      if (!is_candidate_sorted(lh.x, lh.y)) continue;
      const uint32_t pos = nd.n - s.vcnt[(size_t)w * 64 + f] - 1;
      int64_t sl = 0, sr = 0;
      for (uint32_t c = lane; c < C; c += 32) {
        const int64_t r = s.vcls[((size_t)w * v.n_features + f) * C + c];
        const int64_t l = (int64_t)lists.tot[(size_t)w * C + c] - r;
        sl += l * l;
        sr += r * r;
      }
      sl = warp_sum_i64(sl);
      sr = warp_sum_i64(sr);
      const double nl = (double)(pos + 1);
      const double gl = gini_part(sl, nl, nn);
      const double gr = gini_part(sr, __dsub_rn(nn, nl), nn);
      const double sc = __dadd_rn(gl, gr);
      if (sc < best || (sc == best && (f < bf || (f == bf && pos < bp)))) {
        best = sc;
        bf = f;
        bp = pos;
        il = __double2float_rn(gl);
        ir = __double2float_rn(gr);
      }
    }
  }
  if (lane == 0) {
    ct_split_result r;
    r.n_selected = s.nsel[w];
    if (best < dinf()) {
      r.score = best;
      r.feature = bf;
      r.pos = bp;
      r.imp_left = il;
      r.imp_right = ir;
      if (is_virtual(v, bf)) {
        const float2 lh = v.vval[bf];
        r.threshold = midpoint(lh.x, lh.y);
      } else {
        const ct_node nd = lists.nodes[w];
        const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, bf) + nd.start;
        const float* xf = v.x_fm + (size_t)bf * v.n_rows;
        r.threshold = midpoint(xf[entry_row(v, lst[bp])], xf[entry_row(v, lst[bp + 1])]);
      }
    } else {
      r.score = dinf();
      r.feature = NONE;
      r.pos = 0;
      r.imp_left = 0.f;
      r.imp_right = 0.f;
      r.threshold = 0.f;
    }
    s.result[w] = r;
  }
}

template <typename IdxT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_split_reduce(View v, LevelScratch s) {
  const uint32_t count = live_count(s, s.ctr->n_nodes, s.cap_nodes);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_REDUCE], [&](uint32_t w) { split_reduce_item<IdxT, Q>(v, sl, s, w); });
}

// ------------------------------------------------------------------------
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void plan_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                          const TreeView& tv, uint32_t w) {
  const uint32_t lane = lane_id();
  const ct_node nd = lists.nodes[w];
  CT_JOB_VIEW(v, vb, nd.slot);
  const ct_split_result r = s.result[w];
  uint32_t split = r.feature != NONE;
  uint32_t children = 0;
  if (lane == 0 && tv.enabled) {
    const size_t off = (size_t)(nd.slot + tv.slot_base) * tv.capacity;
    if (split) {
      const uint32_t c = atomicAdd(&tv.n_nodes[nd.slot + tv.slot_base], 2u);
      if (c + 2ull > tv.capacity) {
        atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
        split = 0;
      } else {
        children = c;
        tv.left[off + nd.raw_id] = c;
        tv.right[off + nd.raw_id] = c + 1;
        tv.feature[off + nd.raw_id] = r.feature;
        tv.threshold[off + nd.raw_id] = r.threshold;
        tv.value[off + nd.raw_id] = 0;
      }
    }
    if (!split) {
      const IdxT* l0 = list_ptr<IdxT>(v, nd.buf, nd.slot, 0) + nd.start;
      tv.left[off + nd.raw_id] = 0;
      tv.right[off + nd.raw_id] = 0;
      tv.feature[off + nd.raw_id] = 0;
      tv.threshold[off + nd.raw_id] = 0.f;
      tv.value[off + nd.raw_id] = entry_label<LabT>(v, l0[0]);
    }
  }
  split = __shfl_sync(FULL, split, 0);
  children = __shfl_sync(FULL, children, 0);
  if (!split) return;
  const uint32_t npp = ceil_div(nd.n, PART_PIECE);
  const bool big = nd.n > s.small_rows;
  const bool huge = big && nd.n >= s.huge_rows && s.huge_segs && huge_partition_ok(v.bit_words);
  const uint32_t ntiles = big ? ceil_div(nd.n, TILE_ELEMS) : 0u;
  const uint64_t* nmask = lists.node_mask ? lists.node_mask + (size_t)w * v.mask_stride : nullptr;
  const uint64_t skip = (nmask ? nmask[0] : 0ull) | virtual_skip(v);
  const uint64_t* skip_hi = nmask && v.n_features > 64 ? nmask + 1 : nullptr;
  // features whose lists move
  uint32_t nskip = (uint32_t)__popcll(skip);
  if (skip_hi)
    for (uint32_t k = 0; k + 1 < mask_words(v.n_features); ++k) nskip += (uint32_t)__popcll(skip_hi[k]);
  const uint32_t nact = v.n_features - nskip;
  uint32_t sidx = 0, pbase = 0, tbase = 0, gidx = 0, ok = 1;
  if (lane == 0) {
    sidx = atomicAdd(&s.ctr->n_splits, 1u);
    atomicAdd(&s.ctr->split_total, (unsigned long long)nd.n);
    atomicAdd(&s.ctr->part_elems, (unsigned long long)nd.n * nact);
    pbase = atomicAdd(&s.ctr->n_part_pieces, npp);
    if (big) {
      gidx = atomicAdd(huge ? &s.ctr->n_huge_segs : &s.ctr->n_big_segs, 1u);
      tbase = atomicAdd(&s.ctr->n_tiles, ntiles);
    } else {
      gidx = atomicAdd(&s.ctr->n_small_segs, 1u);
    }
    if (sidx >= s.cap_nodes || gidx >= (huge ? s.cap_huge : s.cap_nodes) || pbase + (uint64_t)npp > s.cap_part ||
        (big && tbase + (uint64_t)ntiles > s.cap_status)) {
      atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
      ok = 0;
    } else {
      SplitRec sr;
      sr.node = w;
      sr.feature = r.feature;
      sr.pos = r.pos;
      sr.children = children;
      s.splits[sidx] = sr;
      PartSeg sg;
      sg.in = list_ptr<IdxT>(v, nd.buf, nd.slot, 0) + nd.start;
      sg.out = list_ptr<IdxT>(v, nd.buf ^ 1u, nd.slot, 0) + nd.start;
      sg.bits = slot_bits(v, nd.slot);
      sg.in_fstride = v.stride;
      sg.out_fstride = v.stride;
      sg.n_features = v.n_features;
      sg.row_mask = v.row_mask;
      sg.n = nd.n;
      sg.nl = r.pos + 1;
      sg.status = tbase;
      sg.skip = skip;
      sg.skip_hi = skip_hi;
      (huge ? s.huge_segs : big ? s.big_segs : s.small_segs)[gidx] = sg;
    }
  }
  ok = __shfl_sync(FULL, ok, 0);
  if (!ok) return;
  sidx = __shfl_sync(FULL, sidx, 0);
  pbase = __shfl_sync(FULL, pbase, 0);
  tbase = __shfl_sync(FULL, tbase, 0);
  gidx = __shfl_sync(FULL, gidx, 0);
  for (uint32_t c = lane; c < v.n_classes; c += 32) s.split_left[(size_t)sidx * v.n_classes + c] = 0;
  for (uint32_t j = lane; j < npp; j += 32) {
    PartPiece pp;
    pp.split = sidx;
    pp.j = j;
    pp.npieces = npp;
    pp.status = 0;
    s.part[pbase + j] = pp;
  }
  for (uint32_t j = lane; j < ntiles; j += 32) {
    PartTile tl;
    tl.seg = gidx;
    tl.j = j;
    tl.ntiles = ntiles;
    tl.pad = 0;
    s.tiles[tbase + j] = tl;
  }
  if (big) {
    // the segment's active chains (features whose lists move): k_part_big and
    // k_part_seg claim these instead of every (segment, feature); a huge
    // segment's are padded to a multiple of four so that k_part_seg's quads
    // never span two segments
    const uint32_t F = v.n_features;
    const uint32_t nlist = huge ? (nact + 3u) & ~3u : nact;
    uint32_t* count = huge ? &s.ctr->n_hchains : &s.ctr->n_bchains;
    uint2* list = huge ? s.hchains : s.bchains;
    const uint32_t cap = huge ? s.cap_hchains : s.cap_bchains;
    uint32_t hb = 0;
    if (lane == 0) {
      hb = atomicAdd(count, nlist);
      if (hb + (uint64_t)nlist > cap) {
        atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
        hb = NONE;
      }
    }
    hb = __shfl_sync(FULL, hb, 0);
    if (hb == NONE) return;
    uint32_t done = 0;
    for (uint32_t f0 = 0; f0 < F; f0 += 32) {
      const uint32_t f = f0 + lane;
      const bool act = f < F && !(f < 64 ? masked(skip, f) : mask_bit(skip_hi, f - 64));
      const unsigned am = __ballot_sync(FULL, act);
      if (act) list[hb + done + __popc(am & lanemask_lt())] = make_uint2(gidx, f);
      done += __popc(am);
    }
    for (uint32_t i = nact + lane; i < nlist; i += 32) list[hb + i] = make_uint2(gidx, NONE);
  }
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_plan(View v, LevelScratch s, TreeView tv) {
  const uint32_t count = live_count(s, s.ctr->n_nodes, s.cap_nodes);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_PLAN], [&](uint32_t w) { plan_item<IdxT, LabT, Q>(v, sl, s, tv, w); });
}

// ------------------------------------------------------------------------
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void fill_mark_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                               uint32_t* cnt, uint32_t pi) {
  const uint32_t C = vb.n_classes;
  const uint32_t lane = lane_id();
  const PartPiece pp = s.part[pi];
  const SplitRec sr = s.splits[pp.split];
  const ct_node nd = lists.nodes[sr.node];
  CT_JOB_VIEW(v, vb, nd.slot);
  // a virtual split feature: its left rows are the node's rows with its low
  // value, read from the row list (row order) and the rows' value bits
  const bool virt = is_virtual(v, sr.feature);
  const IdxT* lst = list_ptr<IdxT>(v, nd.buf, nd.slot, virt ? v.vslot : sr.feature) + nd.start;
  uint32_t* bw = slot_bits(v, nd.slot);
  for (uint32_t c = lane; c < C; c += 32) cnt[c] = 0;
  __syncwarp();
  const uint32_t lo = pp.j * PART_PIECE;
  const uint32_t hi = min(lo + PART_PIECE, nd.n);
  // all the piece's index loads first, then the mark bits: every row of a
  // split node is set (left) or cleared (right) once per step, by an atomic
  // on its 32-row word, so no byte table is packed afterwards
  uint32_t rows[PART_ROUNDS], cls[PART_ROUNDS];
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    const uint32_t p = lo + r * 32 + lane;
    rows[r] = p < hi ? (uint32_t)__ldcs(lst + p) : 0u;
  }
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    const uint32_t p = lo + r * 32 + lane;
    cls[r] = NONE;
    if (p < hi) {
      const uint32_t row = entry_row(v, rows[r]);
      const bool left = virt ? !((__ldg(v.vrow + row) >> sr.feature) & 1ull) : p <= sr.pos;
      if (left) atomicOr(bw + (row >> 5), 1u << (row & 31));
      else if (Q) atomicAnd(bw + (row >> 5), ~(1u << (row & 31)));
      if (left) cls[r] = entry_label<LabT>(v, rows[r]);
    }
  }
#pragma unroll
  for (uint32_t r = 0; r < PART_ROUNDS; ++r) {
    if (lo + r * 32 >= hi) break;
    const uint32_t c = cls[r];
    const unsigned grp = __match_any_sync(FULL, c);
    if (c != NONE && (grp >> lane) == 1u) cnt[c] += __popc(grp);
    __syncwarp();
  }
  uint32_t* out = s.split_left + (size_t)pp.split * C;
  for (uint32_t c = lane; c < C; c += 32)
    if (cnt[c]) atomicAdd(&out[c], cnt[c]);
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK) k_fill_mark(View v, LevelScratch s) {
  extern __shared__ uint32_t smem[];
  uint32_t* cnt = smem + (threadIdx.x >> 5) * v.n_classes;
  const uint32_t count = live_count(s, s.ctr->n_part_pieces, s.cap_part);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_FILL], [&](uint32_t pi) { fill_mark_item<IdxT, LabT, Q>(v, sl, s, cnt, pi); });
}

// ------------------------------------------------------------------------
template <typename IdxT, typename LabT, bool Q>
__device__ __forceinline__ void children_item(const View& vb, const StepLists& lists, const LevelScratch& s,
                                              const TreeView& tv, uint32_t cap_next, uint32_t small_cut,
                                              ct_node* small, uint32_t cap_small, uint32_t w) {
  const uint32_t lane = lane_id();
  const uint32_t* tot = lists.tot;
  ct_node* next = lists.next;
  uint32_t* next_tot = lists.next_tot;
  const SplitRec sr = s.splits[w];
  const ct_node nd = lists.nodes[sr.node];
  CT_JOB_VIEW(v, vb, nd.slot);
  const ct_split_result r = s.result[sr.node];
  const uint32_t nl = sr.pos + 1;
  const uint32_t C = v.n_classes;
  for (int side = 0; side < 2; ++side) {
    ct_node ch;
    ch.slot = nd.slot;
    ch.n = side ? nd.n - nl : nl;
    ch.start = side ? nd.start + nl : nd.start;
    ch.raw_id = sr.children + side;
    ch.key = child_key(nd.key, side);
    ch.impurity = side ? r.imp_right : r.imp_left;
    ch.buf = nd.buf ^ 1u;
    const bool leaf = ch.impurity == 0.0f || ch.n < v.mss;
    if (leaf) {
      if (lane == 0 && tv.enabled) {
        const size_t off = (size_t)(nd.slot + tv.slot_base) * tv.capacity + ch.raw_id;
        const IdxT* l0 = list_ptr<IdxT>(v, ch.buf, ch.slot, 0) + ch.start;
        tv.left[off] = 0;
        tv.right[off] = 0;
        tv.feature[off] = 0;
        tv.threshold[off] = 0.f;
        tv.value[off] = entry_label<LabT>(v, l0[0]);
      }
      continue;
    }
    if (small_cut != 0 && ch.n <= small_cut) {
      uint32_t placed = 0;
      if (lane == 0) {
        const uint32_t idx = atomicAdd(&s.ctr->n_small, 1u);
        if (idx < cap_small) {
          small[idx] = ch;
          atomicAdd(&s.ctr->small_total, (unsigned long long)ch.n);
          placed = 1;
        }
      }
      if (__shfl_sync(FULL, placed, 0)) continue;
      // the subtree list is full: the level steps split this child
    }
    uint32_t idx = 0;
    if (lane == 0) {
      idx = atomicAdd(&s.ctr->n_next, 1u);
      if (idx < cap_next) {
        next[idx] = ch;
        atomicAdd(&s.ctr->next_total, (unsigned long long)ch.n);
      } else {
        atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
      }
    }
    idx = __shfl_sync(FULL, idx, 0);
    if (idx >= cap_next) continue;
    for (uint32_t c = lane; c < C; c += 32) {
      const uint32_t left = s.split_left[(size_t)w * C + c];
      next_tot[(size_t)idx * C + c] = side ? tot[(size_t)sr.node * C + c] - left : left;
    }
    if (lists.next_mask) {
      // the child's constant features: the parent's, and those whose values
      // agree at the child's first and last positions (the child's lists of
      // the others were just partitioned); one mask word per 64 features
      const uint32_t mw = mask_words(v.n_features);
      const uint32_t stride = Q ? v.mask_stride : mw;  // equal in a fit of one job
      const uint64_t* pm = lists.node_mask + (size_t)sr.node * stride;
      uint64_t* cmw = lists.next_mask + (size_t)idx * stride;
      for (uint32_t k = 0; k < mw; ++k) {
        const uint64_t pw = pm[k];
        uint64_t cw = pw;
#pragma unroll
        for (uint32_t h = 0; h < 2; ++h) {
          const uint32_t f = k * 64 + h * 32 + lane;
          bool cst = false;
          if (f > 0 && f < v.n_features && !((pw >> (f & 63)) & 1u) && !is_virtual(v, f)) {
            const IdxT* lst = list_ptr<IdxT>(v, ch.buf, ch.slot, f) + ch.start;
            const float* xf = v.x_fm + (size_t)f * v.n_rows;
            cst = xf[entry_row(v, lst[0])] == xf[entry_row(v, lst[ch.n - 1])];
          }
          cw |= (uint64_t)__ballot_sync(FULL, cst) << (h * 32);
        }
        if (lane == 0) cmw[k] = cw;
      }
    }
  }
}

template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK)
k_children(View v, LevelScratch s, TreeView tv, uint32_t cap_next, uint32_t small_cut, ct_node* small,
           uint32_t cap_small) {
  const uint32_t count = live_count(s, s.ctr->n_splits, s.cap_nodes);
  const StepLists sl = *s.step;
  for_items(count, &s.ctr->claim[ITEM_CHILDREN], [&](uint32_t w) {
    children_item<IdxT, LabT, Q>(v, sl, s, tv, cap_next, small_cut, small, cap_small, w);
  });
}

// ------------------------------------------------------------------------
// Warp subtrees.  A node of at most 32 rows is grown to its leaves by one
// warp, one row per lane, without partitioning any feature list: below such
// a node, re-partitioning all F lists every level costs far more than the m
// features each node scans.  The rows are read from feature 0's list, so
// lane order is feature-0 order and a node's leaf label is the label of its
// lowest lane (the first-row rule of the level steps).  A sub-node is a mask
// of lanes.  Per node the selected features are those of k_select (first m
// non-constant ones of the node's permutation); each is sorted across the
// lanes by (value, row) with a bitonic network, the sorted order the index
// lists hold, and scanned with the arithmetic of k_split_scan; the best is the
// lowest (score, feature id, position).  Pending nodes sit on a per-warp
// stack in shared memory; raw node ids come from the tree's node counter
// (the host renumbers breadth-first), so the trees are the level steps' trees.
struct SubEntry {
  uint32_t mask;
  uint32_t raw;
  uint64_t key;
};

__device__ __forceinline__ uint64_t warp_sort_u64(uint64_t v, uint32_t lane) {
#pragma unroll
  for (uint32_t k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      const uint64_t o = __shfl_xor_sync(FULL, v, j);
      const bool up = (lane & k) == 0u;
      const bool lo = (lane & j) == 0u;
      v = (lo == up) ? (o < v ? o : v) : (o > v ? o : v);
    }
  }
  return v;
}

template <typename IdxT, typename LabT>
__device__ __forceinline__ void subtree_leaf(const View& v, const TreeView& tv, size_t toff, uint32_t raw,
                                             uint32_t mask, uint32_t lab, uint32_t lane) {
  const uint32_t value = __shfl_sync(FULL, lab, __ffs(mask) - 1);
  if (lane == 0) {
    tv.left[toff + raw] = 0;
    tv.right[toff + raw] = 0;
    tv.feature[toff + raw] = 0;
    tv.threshold[toff + raw] = 0.f;
    tv.value[toff + raw] = value;
  }
}

// One row per lane: grows the subtree of `cur` (lanes in feature-0 order,
// row ids and labels in registers; lanes outside the node carry NONE).
template <typename IdxT, typename LabT>
__device__ void grow_small(const View& v, const LevelScratch& s, const TreeView& tv, uint32_t tslot, size_t toff,
                           uint32_t row, uint32_t lab, SubEntry cur, SubEntry* stack, uint32_t lane) {
  const uint32_t F = v.n_features, m = v.max_features;
  const unsigned lt = lanemask_lt();
  int sp = 0;
  while (true) {
    const uint32_t mask = cur.mask;
    const uint32_t n = __popc(mask);
    const bool in = (mask >> lane) & 1u;
    // class totals of the node: Σ_c T_c² as a sum over its rows of T_(c(row))
    const uint32_t tcls = __popc(__match_any_sync(FULL, in ? lab : NONE));
    const int64_t sr0 = (int64_t)warp_sum_u32(in ? tcls : 0u);
    const double nn = (double)n;
    double best = dinf();
    uint32_t bf = NONE, bp = 0, bmask = 0;
    float bil = 0.f, bir = 0.f, bthr = 0.f;
    uint32_t taken = 0;
    // the next feature's values are gathered while the current one is sorted and scanned
    uint32_t f_nx = feature_perm(0, F, cur.key, v.feistel_h);
    float x_nx = in ? v.x_fm[(size_t)f_nx * v.n_rows + row] : 0.f;
    for (uint32_t i = 0; i < F && taken < m; ++i) {
      const uint32_t f = f_nx;
      const float* xf = v.x_fm + (size_t)f * v.n_rows;
      const float xv = x_nx;
      if (i + 1 < F) {
        f_nx = feature_perm(i + 1, F, cur.key, v.feistel_h);
        x_nx = in ? v.x_fm[(size_t)f_nx * v.n_rows + row] : 0.f;
      }
      const uint32_t ord = f32_order(xv);
      if (__reduce_min_sync(FULL, in ? ord : 0xffffffffu) == __reduce_max_sync(FULL, in ? ord : 0u)) continue;
      ++taken;
      const uint64_t key = in ? ((uint64_t)ord << 32) | ((uint64_t)row << 5) | lane : ~0ull;
      const uint64_t sk = warp_sort_u64(key, lane);  // lane p holds sorted position p
      const bool valid = lane < n;
      const uint32_t src = (uint32_t)sk & 31u;
      const uint32_t srow = (uint32_t)sk >> 5;
      const uint32_t cl = __shfl_sync(FULL, lab, src);
      const uint32_t c = valid ? cl : NONE;
      const float x = f32_unorder((uint32_t)(sk >> 32));
      const float xn = __shfl_down_sync(FULL, x, 1);
      const unsigned grp = __match_any_sync(FULL, c);
      const int32_t k = (int32_t)__popc(grp & lt);
      const int32_t tc = (int32_t)__popc(grp);
      const int32_t il = warp_incl_scan_i32(valid ? 2 * k + 1 : 0);
      const int32_t ir = warp_incl_scan_i32(valid ? 1 - 2 * (tc - k) : 0);
      double sc = dinf();
      float gil = 0.f, gir = 0.f;
      if (valid && lane + 1 < n && is_candidate_sorted(x, xn)) {
        const double nl = (double)(lane + 1);
        const double nr = __dsub_rn(nn, nl);
        const double gl = gini_part((int64_t)il, nl, nn);
        const double gr = gini_part(sr0 + (int64_t)ir, nr, nn);
        sc = __dadd_rn(gl, gr);
        gil = __double2float_rn(gl);
        gir = __double2float_rn(gr);
      }
      uint32_t pos = lane;
      warp_argmin2(sc, pos, gil, gir);
      if (sc < dinf() && (sc < best || (sc == best && f < bf))) {
        best = sc;
        bf = f;
        bp = pos;
        bil = gil;
        bir = gir;
        bmask = __reduce_or_sync(FULL, (valid && lane <= pos) ? (1u << src) : 0u);
        const uint32_t r0 = __shfl_sync(FULL, srow, pos);
        const uint32_t r1 = __shfl_sync(FULL, srow, (pos + 1) & 31u);
        bthr = midpoint(xf[r0], xf[r1]);
      }
    }
    bool split = bf != NONE;
    uint32_t c0 = 0;
    if (split && lane == 0) {
      c0 = atomicAdd(&tv.n_nodes[tslot], 2u);
      if (c0 + 2ull > tv.capacity) {
        atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
        split = false;
      }
    }
    split = __shfl_sync(FULL, split, 0);
    c0 = __shfl_sync(FULL, c0, 0);
    if (!split) {
      subtree_leaf<IdxT, LabT>(v, tv, toff, cur.raw, mask, lab, lane);
    } else {
      if (lane == 0) {
        tv.left[toff + cur.raw] = c0;
        tv.right[toff + cur.raw] = c0 + 1;
        tv.feature[toff + cur.raw] = bf;
        tv.threshold[toff + cur.raw] = bthr;
        tv.value[toff + cur.raw] = 0;
      }
      const uint32_t masks[2] = {bmask, mask & ~bmask};
      const float imps[2] = {bil, bir};
      for (int side = 0; side < 2; ++side) {
        const uint32_t cm = masks[side];
        if (imps[side] == 0.0f || __popc(cm) < v.mss) {
          subtree_leaf<IdxT, LabT>(v, tv, toff, c0 + side, cm, lab, lane);
        } else if (sp < 33) {
          if (lane == 0) stack[sp] = SubEntry{cm, c0 + (uint32_t)side, child_key(cur.key, side)};
          ++sp;
        } else {
          if (lane == 0) atomicOr(&s.ctr->error, DEV_ERR_INTERNAL);
        }
      }
    }
    __syncwarp();
    if (sp == 0) break;
    --sp;
    cur = stack[sp];
    __syncwarp();
  }
}

// Four rows per lane, for subtree roots of 33..128 rows.  Slot s (lane
// s % 32, register s / 32) holds the root's s-th row in feature-0 order, so
// a node's leaf label is its lowest slot's; the sort key carries each slot's
// rank by row id, so equal values still order by row id.  A node is a
// 128-bit mask of slots; a child of at most 32 rows is compacted onto the
// lanes (slot order) and handed to grow_small.
constexpr uint32_t WIDE_ROWS = 128;
constexpr uint32_t WIDE_STACK = 4;  // pending nodes of > 32 rows are disjoint: at most 3
struct WideEntry {
  uint32_t m[4];
  uint32_t raw;
  uint32_t pad;
  uint64_t key;
};

// Shared memory of one warp of k_subtree, in words: rows, labels and row
// ranks of 128 slots, two class arrays, then the two stacks (8-byte fields)
// at a 16-byte boundary; the whole region is a multiple of 16 bytes, so every
// warp's stacks stay aligned.
__host__ __device__ __forceinline__ uint32_t subtree_stacks_word(uint32_t n_classes) {
  return (3 * WIDE_ROWS + 2 * n_classes + 3u) & ~3u;
}
__host__ __device__ __forceinline__ uint32_t subtree_warp_words(uint32_t n_classes) {
  return subtree_stacks_word(n_classes) + WIDE_STACK * (uint32_t)(sizeof(WideEntry) / 4) +
         33u * (uint32_t)(sizeof(SubEntry) / 4);
}

// Bitonic network over 128 keys, element lane + 32 k in register k.
__device__ __forceinline__ void warp_sort128(uint64_t (&v)[4], uint32_t lane) {
#pragma unroll
  for (uint32_t size = 2; size <= WIDE_ROWS; size <<= 1) {
#pragma unroll
    for (uint32_t j = size >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const uint32_t kj = j >> 5;
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
          if (k & kj) continue;
          const uint32_t k2 = k | kj;
          const bool up = ((lane + 32 * k) & size) == 0u;
          const uint64_t a = v[k], b = v[k2];
          const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
          v[k] = up ? lo : hi;
          v[k2] = up ? hi : lo;
        }
      } else {
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
          const uint64_t o = __shfl_xor_sync(FULL, v[k], j);
          const bool up = ((lane + 32 * k) & size) == 0u;
          const bool lower = (lane & j) == 0u;
          v[k] = (lower == up) ? (o < v[k] ? o : v[k]) : (o > v[k] ? o : v[k]);
        }
      }
    }
  }
}

__device__ __forceinline__ uint64_t pick4(const uint64_t (&v)[4], uint32_t k) {
  return k == 0 ? v[0] : k == 1 ? v[1] : k == 2 ? v[2] : v[3];
}

__device__ __forceinline__ uint32_t lowest_slot(const uint32_t (&m)[4]) {
  return m[0] ? __ffs(m[0]) - 1 : m[1] ? 31 + __ffs(m[1]) : m[2] ? 63 + __ffs(m[2]) : 95 + __ffs(m[3]);
}

template <typename IdxT, typename LabT>
__device__ void grow_wide(const View& v, const LevelScratch& s, const TreeView& tv, const ct_node& nd, size_t toff,
                          uint32_t* wsm, uint32_t lane) {
  const uint32_t C = v.n_classes, F = v.n_features, m = v.max_features;
  const uint32_t tslot = nd.slot + tv.slot_base;
  uint32_t* row_s = wsm;
  uint32_t* lab_s = row_s + WIDE_ROWS;
  uint32_t* rr_s = lab_s + WIDE_ROWS;
  uint32_t* cnt = rr_s + WIDE_ROWS;
  uint32_t* T = cnt + C;
  WideEntry* wstack = reinterpret_cast<WideEntry*>(wsm + subtree_stacks_word(C));
  SubEntry* stack1 = reinterpret_cast<SubEntry*>(wstack + WIDE_STACK);
  const unsigned lt = lanemask_lt();
  const uint32_t n0 = nd.n;
  const IdxT* l0 = list_ptr<IdxT>(v, nd.buf, nd.slot, 0) + nd.start;
  uint32_t rowr[4], labr[4], rrr[4];
  uint64_t kk[4];
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) {
    const uint32_t slot = lane + 32 * k;
    const bool have = slot < n0;
    const uint32_t e = have ? (uint32_t)l0[slot] : 0u;
    rowr[k] = have ? entry_row(v, e) : 0u;
    labr[k] = have ? entry_label<LabT>(v, e) : NONE;
    row_s[slot] = rowr[k];
    lab_s[slot] = labr[k];
    kk[k] = have ? ((uint64_t)rowr[k] << 7) | slot : ~0ull;
  }
  warp_sort128(kk, lane);  // position e holds the slot of rank e by row id
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k)
    if (lane + 32 * k < n0) rr_s[(uint32_t)kk[k] & 127u] = lane + 32 * k;
  __syncwarp();
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k) rrr[k] = lane + 32 * k < n0 ? rr_s[lane + 32 * k] : 0u;
  WideEntry cur{};
#pragma unroll
  for (uint32_t k = 0; k < 4; ++k)
    cur.m[k] = n0 >= 32 * (k + 1) ? FULL : (n0 > 32 * k ? (1u << (n0 - 32 * k)) - 1u : 0u);
  cur.raw = nd.raw_id;
  cur.key = nd.key;
  int wsp = 0;
  while (true) {
    bool in[4];
    uint32_t n = 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
      in[k] = (cur.m[k] >> lane) & 1u;
      n += __popc(cur.m[k]);
    }
    // class totals of the node
    for (uint32_t c = lane; c < C; c += 32) T[c] = 0;
    __syncwarp();
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
      const uint32_t c = in[k] ? labr[k] : NONE;
      const unsigned grp = __match_any_sync(FULL, c);
      if (in[k] && (grp & lt) == 0u) T[c] += __popc(grp);
      __syncwarp();
    }
    uint32_t tsum = 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) tsum += in[k] ? T[labr[k]] : 0u;
    const int64_t sr0 = (int64_t)warp_sum_u32(tsum);
    const double nn = (double)n;
    double best = dinf();
    uint32_t bf = NONE, bp = 0, bm[4] = {0u, 0u, 0u, 0u};
    float bil = 0.f, bir = 0.f, bthr = 0.f;
    uint32_t taken = 0;
    uint32_t f_nx = feature_perm(0, F, cur.key, v.feistel_h);
    float x_nx[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) x_nx[k] = in[k] ? v.x_fm[(size_t)f_nx * v.n_rows + rowr[k]] : 0.f;
    for (uint32_t i = 0; i < F && taken < m; ++i) {
      const uint32_t f = f_nx;
      const float* xf = v.x_fm + (size_t)f * v.n_rows;
      uint32_t ord[4];
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) ord[k] = f32_order(x_nx[k]);
      if (i + 1 < F) {
        f_nx = feature_perm(i + 1, F, cur.key, v.feistel_h);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) x_nx[k] = in[k] ? v.x_fm[(size_t)f_nx * v.n_rows + rowr[k]] : 0.f;
      }
      uint32_t lmin = 0xffffffffu, lmax = 0u;
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        if (in[k]) {
          lmin = min(lmin, ord[k]);
          lmax = max(lmax, ord[k]);
        }
      if (__reduce_min_sync(FULL, lmin) == __reduce_max_sync(FULL, lmax)) continue;
      ++taken;
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        kk[k] = in[k] ? ((uint64_t)ord[k] << 32) | ((uint64_t)rrr[k] << 7) | (lane + 32 * k) : ~0ull;
      warp_sort128(kk, lane);  // position lane + 32 k
      for (uint32_t c = lane; c < C; c += 32) cnt[c] = 0;
      __syncwarp();
      int64_t sl = 0, sr = sr0;
      double bsc = dinf();
      uint32_t bpos = NONE;
      float bgl = 0.f, bgr = 0.f;
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        const uint32_t p = lane + 32 * k;
        const bool valid = p < n;
        const uint32_t slot = (uint32_t)kk[k] & 127u;
        const uint32_t c = valid ? lab_s[slot] : NONE;
        const float x = f32_unorder((uint32_t)(kk[k] >> 32));
        float xn = __shfl_down_sync(FULL, x, 1);
        const float first_next = __shfl_sync(FULL, k + 1 < 4 ? f32_unorder((uint32_t)(kk[k + 1 < 4 ? k + 1 : k] >> 32)) : 0.f, 0);
        if (lane == 31) xn = first_next;
        const unsigned grp = __match_any_sync(FULL, c);
        const int32_t kr = valid ? (int32_t)(cnt[c] + __popc(grp & lt)) : 0;
        const int32_t tc = valid ? (int32_t)T[c] : 0;
        __syncwarp();
        if (valid && (grp & lt) == 0u) cnt[c] += __popc(grp);
        __syncwarp();
        const int32_t il = warp_incl_scan_i32(valid ? 2 * kr + 1 : 0);
        const int32_t ir = warp_incl_scan_i32(valid ? 1 - 2 * (tc - kr) : 0);
        const int64_t SL = sl + il, SR = sr + ir;
        sl += __shfl_sync(FULL, il, 31);
        sr += __shfl_sync(FULL, ir, 31);
        if (valid && p + 1 < n && is_candidate_sorted(x, xn)) {
          const double nl = (double)(p + 1);
          const double nr = __dsub_rn(nn, nl);
          const double gl = gini_part(SL, nl, nn);
          const double gr = gini_part(SR, nr, nn);
          const double sc = __dadd_rn(gl, gr);
          if (sc < bsc) {
            bsc = sc;
            bpos = p;
            bgl = __double2float_rn(gl);
            bgr = __double2float_rn(gr);
          }
        }
      }
      warp_argmin2(bsc, bpos, bgl, bgr);
      if (bsc < dinf() && (bsc < best || (bsc == best && f < bf))) {
        best = bsc;
        bf = f;
        bp = bpos;
        bil = bgl;
        bir = bgr;
        uint32_t wb[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
          const uint32_t p = lane + 32 * k;
          const uint32_t slot = (uint32_t)kk[k] & 127u;
          const uint32_t bit = (p < n && p <= bpos) ? (1u << (slot & 31u)) : 0u;
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) wb[q] |= (slot >> 5) == q ? bit : 0u;
        }
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) bm[q] = __reduce_or_sync(FULL, wb[q]);
        const uint32_t s0 = (uint32_t)__shfl_sync(FULL, pick4(kk, bpos >> 5), bpos & 31u) & 127u;
        const uint32_t s1 = (uint32_t)__shfl_sync(FULL, pick4(kk, (bpos + 1) >> 5), (bpos + 1) & 31u) & 127u;
        bthr = midpoint(xf[row_s[s0]], xf[row_s[s1]]);
      }
    }
    bool split = bf != NONE;
    uint32_t c0 = 0;
    if (split && lane == 0) {
      c0 = atomicAdd(&tv.n_nodes[tslot], 2u);
      if (c0 + 2ull > tv.capacity) {
        atomicOr(&s.ctr->error, DEV_ERR_CAPACITY);
        split = false;
      }
    }
    split = __shfl_sync(FULL, split, 0);
    c0 = __shfl_sync(FULL, c0, 0);
    if (!split) {
      if (lane == 0) {
        tv.left[toff + cur.raw] = 0;
        tv.right[toff + cur.raw] = 0;
        tv.feature[toff + cur.raw] = 0;
        tv.threshold[toff + cur.raw] = 0.f;
        tv.value[toff + cur.raw] = lab_s[lowest_slot(cur.m)];
      }
    } else {
      if (lane == 0) {
        tv.left[toff + cur.raw] = c0;
        tv.right[toff + cur.raw] = c0 + 1;
        tv.feature[toff + cur.raw] = bf;
        tv.threshold[toff + cur.raw] = bthr;
        tv.value[toff + cur.raw] = 0;
      }
      const float imps[2] = {bil, bir};
      const uint64_t pkey = cur.key;
      for (int side = 0; side < 2; ++side) {
        uint32_t cm[4];
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) cm[q] = side ? cur.m[q] & ~bm[q] : bm[q];
        const uint32_t nc = __popc(cm[0]) + __popc(cm[1]) + __popc(cm[2]) + __popc(cm[3]);
        const uint32_t raw = c0 + (uint32_t)side;
        if (imps[side] == 0.0f || nc < v.mss) {
          if (lane == 0) {
            tv.left[toff + raw] = 0;
            tv.right[toff + raw] = 0;
            tv.feature[toff + raw] = 0;
            tv.threshold[toff + raw] = 0.f;
            tv.value[toff + raw] = lab_s[lowest_slot(cm)];
          }
        } else if (nc <= 32) {
          // lane i takes the child's i-th slot (slot order = feature-0 order)
          uint32_t row = 0, lab = NONE;
          uint32_t before = 0;
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t c = __popc(cm[q]);
            if (lane >= before && lane < before + c) {
              const uint32_t slot = 32 * q + __fns(cm[q], 0, (int)(lane - before + 1));
              row = row_s[slot];
              lab = lab_s[slot];
            }
            before += c;
          }
          const SubEntry e{nc >= 32 ? FULL : ((1u << nc) - 1u), raw, child_key(pkey, side)};
          grow_small<IdxT, LabT>(v, s, tv, tslot, toff, row, lab, e, stack1, lane);
        } else if (wsp < (int)WIDE_STACK) {
          if (lane == 0) {
            WideEntry e{};
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) e.m[q] = cm[q];
            e.raw = raw;
            e.key = child_key(pkey, side);
            wstack[wsp] = e;
          }
          ++wsp;
        } else {
          if (lane == 0) atomicOr(&s.ctr->error, DEV_ERR_INTERNAL);
        }
      }
    }
    __syncwarp();
    if (wsp == 0) break;
    --wsp;
    cur = wstack[wsp];
    __syncwarp();
  }
}



// Subtree roots of at most 32 rows (the others are skipped).
template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK)
k_subtree(View vb, const ct_node* __restrict__ small, LevelScratch s, TreeView tv, uint32_t cap_small) {
  __shared__ SubEntry stack_all[WARPS_PER_BLOCK][33];
  const uint32_t lane = lane_id();
  const uint32_t count = live_count(s, s.ctr->n_small, cap_small);
  for_items(count, &s.ctr->claim[ITEM_SUBTREE], [&](uint32_t w) {
    const ct_node nd = small[w];
    if (nd.n > 32) return;
    CT_JOB_VIEW(v, vb, nd.slot);
    const size_t toff = (size_t)(nd.slot + tv.slot_base) * tv.capacity;
    const IdxT* l0 = list_ptr<IdxT>(v, nd.buf, nd.slot, 0) + nd.start;
    const bool have = lane < nd.n;
    const uint32_t e = have ? (uint32_t)l0[lane] : 0u;
    const uint32_t row = have ? entry_row(v, e) : 0u;
    const uint32_t lab = have ? entry_label<LabT>(v, e) : NONE;
    const SubEntry cur{nd.n >= 32 ? FULL : ((1u << nd.n) - 1u), nd.raw_id, nd.key};
    grow_small<IdxT, LabT>(v, s, tv, nd.slot + tv.slot_base, toff, row, lab, cur, stack_all[threadIdx.x >> 5],
                           lane);
  });
}

// Subtree roots of 33..128 rows (the others are skipped).
template <typename IdxT, typename LabT, bool Q>
__global__ void __launch_bounds__(THREADS_PER_BLOCK)
k_subtree_wide(View vb, const ct_node* __restrict__ small, LevelScratch s, TreeView tv, uint32_t cap_small) {
  extern __shared__ __align__(16) uint32_t sub_smem[];
  const uint32_t lane = lane_id();
  const uint32_t count = live_count(s, s.ctr->n_small, cap_small);
  uint32_t* wsm = sub_smem + (threadIdx.x >> 5) * subtree_warp_words(vb.n_classes);
  for_items(count, &s.ctr->claim[ITEM_SUBTREE_WIDE], [&](uint32_t w) {
    const ct_node nd = small[w];
    if (nd.n <= 32) return;
    CT_JOB_VIEW(v, vb, nd.slot);
    const size_t toff = (size_t)(nd.slot + tv.slot_base) * tv.capacity;
    grow_wide<IdxT, LabT>(v, s, tv, nd, toff, wsm, lane);
  });
}

__global__ void k_reset_step(Counters* c, uint32_t n_nodes, StepLists* step, StepLists lists) {
  reset_step_counters(c, n_nodes);
  *step = lists;
}

inline uint32_t clamp32(uint64_t x) { return x > 0xffffffffull ? 0xffffffffu : (uint32_t)x; }

// Blocks of a warp-per-item launch: one warp per item, or, for a launch that
// must not depend on the item count (persistent), at most the blocks that
// are resident at once, whose warps then loop over the items.
template <typename K>
uint32_t grid_for(K kernel, uint64_t warps, size_t smem, bool persistent) {
  uint32_t cap = 0;
  if (persistent) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, THREADS_PER_BLOCK, smem);
    cap = (uint32_t)std::max(1, sms) * (uint32_t)std::max(1, per);
  }
  return item_blocks(warps, cap);
}

template <typename IdxT, typename LabT, bool Q>
void split_impl(const View& v, const LevelScratch& s, const LevelCaps& caps, uint32_t scan_piece, bool persistent,
                cudaStream_t st) {
  Prof* pf = current_prof();
  const size_t sm1 = (size_t)WARPS_PER_BLOCK * v.n_classes * sizeof(uint32_t);
  if (v.vmask) {  // counts of the virtual features, before the selection reads them
    pf->begin(CT_K_SCAN);
    const size_t smv = (size_t)WARPS_PER_BLOCK * v.n_features * v.n_classes * sizeof(uint32_t);
    k_vpieces<<<grid_for(k_vpieces, caps.nodes, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(v, s);
    k_vcount<IdxT, LabT><<<grid_for(k_vcount<IdxT, LabT>, caps.vpieces, smv, persistent), THREADS_PER_BLOCK, smv,
                           st>>>(v, s);
    pf->end();
    pf->launched(CT_K_SCAN, 2);
  }
  pf->begin(CT_K_SELECT);
  k_select<IdxT, Q><<<grid_for(k_select<IdxT, Q>, caps.nodes, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(v, s);
  pf->end();
  pf->launched(CT_K_SELECT);
  pf->begin(CT_K_SCAN);
  k_scan_hist<IdxT, LabT, Q><<<grid_for(k_scan_hist<IdxT, LabT, Q>, caps.carry, sm1, persistent), THREADS_PER_BLOCK,
                            sm1, st>>>(v, s);
  k_scan_carry<<<grid_for(k_scan_carry, caps.carry, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(s, v.n_classes);
  k_split_scan<IdxT, LabT, Q><<<grid_for(k_split_scan<IdxT, LabT, Q>, caps.scan, 2 * sm1, persistent), THREADS_PER_BLOCK,
                             2 * sm1, st>>>(v, s);
  if (v.fbin)
    k_scan_two_valued<IdxT, LabT, Q><<<grid_for(k_scan_two_valued<IdxT, LabT, Q>, caps.scan, sm1, persistent),
                                    THREADS_PER_BLOCK, sm1, st>>>(v, s);
  pf->end();
  pf->launched(CT_K_SCAN, v.fbin ? 4 : 3);
  pf->begin(CT_K_REDUCE);
  k_split_reduce<IdxT, Q><<<grid_for(k_split_reduce<IdxT, Q>, caps.nodes, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(v, s);
  pf->end();
  pf->launched(CT_K_REDUCE);
}

template <typename IdxT, typename LabT, bool Q>
void partition_impl(const View& v, const LevelScratch& s_all, const LevelCaps& caps, const TreeView& tv,
                    bool persistent, cudaStream_t st) {
  Prof* pf = current_prof();
  // tile/status capacity of this step: its status words are zeroed, its stride is the column stride
  LevelScratch s = s_all;
  s.cap_status = caps.status;
  const size_t sm1 = (size_t)WARPS_PER_BLOCK * v.n_classes * sizeof(uint32_t);
  pf->begin(CT_K_MARK);
  k_plan<IdxT, LabT, Q><<<grid_for(k_plan<IdxT, LabT, Q>, caps.nodes, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(v, s,
                                                                                                            tv);
  k_fill_mark<IdxT, LabT, Q><<<grid_for(k_fill_mark<IdxT, LabT, Q>, caps.part, sm1, persistent), THREADS_PER_BLOCK, sm1,
                            st>>>(v, s);
  pf->launched(CT_K_MARK, 2);
  pf->end();
  pf->begin(CT_K_PARTITION);
  const PartWork w = level_part_work(v, s);
  launch_seg_partition(sizeof(IdxT), w, caps.nodes, caps.status, st);
  pf->end();
  pf->launched(CT_K_PARTITION, 2);
}

template <typename IdxT, typename LabT, bool Q>
void children_impl(const View& v, const LevelScratch& s, const LevelCaps& caps, const TreeView& tv, uint32_t cap_next,
                   uint32_t small_cut, ct_node* small, uint32_t cap_small, bool persistent, cudaStream_t st) {
  Prof* pf = current_prof();
  pf->begin(CT_K_CHILDREN);
  k_children<IdxT, LabT, Q><<<grid_for(k_children<IdxT, LabT, Q>, caps.nodes, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(
      v, s, tv, cap_next, small_cut, small, cap_small);
  pf->end();
  pf->launched(CT_K_CHILDREN);
}

}  // namespace

// ---------------------------------------------------------------------------
LevelCaps level_caps(const View& v, uint32_t scan_piece, LevelBounds b) {
  LevelCaps c;
  const uint64_t m = v.max_features;
  c.nodes = clamp32(b.nodes);
  c.scan = clamp32(m * (b.samples / scan_piece + b.nodes) + 1);
  c.carry = clamp32(m * (2 * b.samples / scan_piece) + 1);
  c.part = clamp32(b.samples / PART_PIECE + b.nodes + 1);
  c.status = clamp32(b.samples / TILE_ELEMS + b.samples / (SMALL_SEG + 1) + 1);  // tiles of big splits
  c.vpieces = clamp32(b.samples / VPIECE + b.nodes + 1);
  c.huge = clamp32(b.samples / HUGE_SEG + 1);
  c.hchains = clamp32((uint64_t)c.huge * (v.n_features + 3));
  c.bchains = clamp32((b.samples / (SMALL_SEG + 1) + 1) * (uint64_t)v.n_features);
  return c;
}

static size_t carve_or_size(Arena& a, const View& v, const LevelCaps& c, LevelScratch* s, bool virt) {
  const size_t C = v.n_classes;
  LevelScratch t;
  t.cap_nodes = c.nodes;
  t.cap_scan = c.scan;
  t.cap_carry = c.carry;
  t.cap_part = c.part;
  t.cap_status = c.status;
  t.ctr = a.take<Counters>(1);
  t.sel = a.take<uint32_t>((size_t)c.nodes * v.max_features);
  t.nsel = a.take<uint32_t>(c.nodes);
  t.piece_base = a.take<uint32_t>(c.nodes);
  t.piece_cnt = a.take<uint32_t>(c.nodes);
  t.pieces = a.take<ScanPiece>(c.scan);
  t.carry = a.take<uint32_t>((size_t)c.carry * C);
  t.carry_piece = a.take<uint32_t>(c.carry);
  t.tv_pieces = a.take<uint32_t>(c.scan);
  t.best = a.take<PieceBest>(c.scan);
  t.result = a.take<ct_split_result>(c.nodes);
  t.splits = a.take<SplitRec>(c.nodes);
  t.split_left = a.take<uint32_t>((size_t)c.nodes * C);
  t.part = a.take<PartPiece>(c.part);
  t.small_segs = a.take<PartSeg>(c.nodes);
  t.big_segs = a.take<PartSeg>(c.nodes);
  const bool huge = huge_partition_ok(v.bit_words);
  t.huge_segs = huge ? a.take<PartSeg>(c.huge) : nullptr;
  t.hchains = huge ? a.take<uint2>(c.hchains) : nullptr;
  t.cap_huge = huge ? c.huge : 0u;
  t.cap_hchains = huge ? c.hchains : 0u;
  t.bchains = a.take<uint2>(c.bchains);
  t.cap_bchains = c.bchains;
  t.tiles = a.take<PartTile>(c.status);
  t.status = a.take<uint64_t>((size_t)c.status * v.n_features);
  t.step = a.take<StepLists>(1);
  t.huge_rows = HUGE_SEG;
  t.part_shape = 0;
  t.small_rows = SMALL_SEG;
  t.vcnt = virt ? a.take<uint32_t>((size_t)c.nodes * 64) : nullptr;
  t.vcls = virt ? a.take<uint32_t>((size_t)c.nodes * v.n_features * C) : nullptr;
  t.vpieces = virt ? a.take<uint2>(c.vpieces) : nullptr;
  t.cap_vpieces = virt ? c.vpieces : 0u;
  if (s) *s = t;
  return a.used;
}

size_t level_scratch_bytes(const View& v, const LevelCaps& c, bool virt) {
  Arena a{nullptr, 0, 0};
  return carve_or_size(a, v, c, nullptr, virt) + 256;
}

bool carve_level_scratch(Arena& a, const View& v, const LevelCaps& c, LevelScratch* s, bool virt) {
  carve_or_size(a, v, c, s, virt);
  return a.ok();
}

bool virtual_possible(const ct_problem* p) {
  return p->n_features >= 2 && p->n_features <= 64 && fit_label_shift(p) != 0 &&
         (uint64_t)p->n_features * p->n_classes <= 2048;
}

#define CT_DISPATCH(IB, LB, CALL)                                   \
  do {                                                              \
    if ((IB) == 2 && (LB) == 1) { CALL(uint16_t, uint8_t); }        \
    else if ((IB) == 2 && (LB) == 2) { CALL(uint16_t, uint16_t); }  \
    else if ((IB) == 4 && (LB) == 1) { CALL(uint32_t, uint8_t); }   \
    else { CALL(uint32_t, uint16_t); }                              \
  } while (0)

uint32_t item_blocks(uint64_t warps, uint32_t grid_cap) {
  uint64_t b = (warps + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK;
  if (b == 0) b = 1;
  if (grid_cap && b > grid_cap) b = grid_cap;
  return (uint32_t)std::min<uint64_t>(b, 0x7fffffffull);
}

// Q: the view is a forest queue's batch view (View::jobs); the kernels of
// one fit are instantiated without the job lookup.
template <bool Q>
int launch_split_q(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b,
                   uint32_t scan_piece, bool persistent, cudaStream_t st) {
  LevelCaps caps = level_caps(v, scan_piece, b);
  caps.scan = min(caps.scan, s.cap_scan);
  caps.carry = min(caps.carry, s.cap_carry);
#define CALL(I, L) split_impl<I, L, Q>(v, s, caps, scan_piece, persistent, st)
  CT_DISPATCH(ib, lb, CALL);
#undef CALL
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}
int launch_split(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b, uint32_t scan_piece,
                 bool persistent, cudaStream_t st) {
  return v.jobs ? launch_split_q<true>(v, ib, lb, s, b, scan_piece, persistent, st)
                : launch_split_q<false>(v, ib, lb, s, b, scan_piece, persistent, st);
}

template <bool Q>
int launch_partition_q(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b,
                       const TreeView& tv, bool persistent, cudaStream_t st) {
  LevelCaps caps = level_caps(v, DEFAULT_SCAN_PIECE, b);
  caps.part = min(caps.part, s.cap_part);
  caps.status = min(caps.status, s.cap_status);
  if (!Q && v.bits) CT_CUDA_TRY(cudaMemsetAsync(v.bits, 0, (size_t)v.n_slots * v.bit_words * sizeof(uint32_t), st));
#define CALL(I, L) partition_impl<I, L, Q>(v, s, caps, tv, persistent, st)
  CT_DISPATCH(ib, lb, CALL);
#undef CALL
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}
int launch_partition(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b,
                     const TreeView& tv, bool persistent, cudaStream_t st) {
  return v.jobs ? launch_partition_q<true>(v, ib, lb, s, b, tv, persistent, st)
                : launch_partition_q<false>(v, ib, lb, s, b, tv, persistent, st);
}

template <bool Q>
int launch_children_q(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b,
                      const TreeView& tv, uint32_t cap_next, uint32_t small_cut, ct_node* small, uint32_t cap_small,
                      bool persistent, cudaStream_t st) {
  LevelCaps caps = level_caps(v, DEFAULT_SCAN_PIECE, b);
#define CALL(I, L) children_impl<I, L, Q>(v, s, caps, tv, cap_next, small_cut, small, cap_small, persistent, st)
  CT_DISPATCH(ib, lb, CALL);
#undef CALL
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}
int launch_children(const View& v, uint32_t ib, uint32_t lb, const LevelScratch& s, LevelBounds b, const TreeView& tv,
                    uint32_t cap_next, uint32_t small_cut, ct_node* small, uint32_t cap_small, bool persistent,
                    cudaStream_t st) {
  return v.jobs ? launch_children_q<true>(v, ib, lb, s, b, tv, cap_next, small_cut, small, cap_small, persistent, st)
                : launch_children_q<false>(v, ib, lb, s, b, tv, cap_next, small_cut, small, cap_small, persistent, st);
}

template <bool Q>
int launch_subtrees_q(const View& v, uint32_t ib, uint32_t lb, const ct_node* small, uint32_t cap_small,
                      uint32_t bound, bool wide, bool persistent, const LevelScratch& s, const TreeView& tv,
                      cudaStream_t st);
int launch_subtrees(const View& v, uint32_t ib, uint32_t lb, const ct_node* small, uint32_t cap_small, uint32_t bound,
                    bool wide, bool persistent, const LevelScratch& s, const TreeView& tv, cudaStream_t st) {
  return v.jobs ? launch_subtrees_q<true>(v, ib, lb, small, cap_small, bound, wide, persistent, s, tv, st)
                : launch_subtrees_q<false>(v, ib, lb, small, cap_small, bound, wide, persistent, s, tv, st);
}

template <bool Q>
int launch_subtrees_q(const View& v, uint32_t ib, uint32_t lb, const ct_node* small, uint32_t cap_small,
                      uint32_t bound, bool wide, bool persistent, const LevelScratch& s, const TreeView& tv,
                      cudaStream_t st) {
  if (cap_small == 0 || bound == 0) return CT_OK;
  Prof* pf = current_prof();
  pf->begin(CT_K_SUBTREE);
  const uint32_t items = std::min(bound, cap_small);
#define CALL(I, L)                                                                                           \
  k_subtree<I, L, Q><<<grid_for(k_subtree<I, L, Q>, items, 0, persistent), THREADS_PER_BLOCK, 0, st>>>(v, small, s, tv, \
                                                                                                cap_small)
  CT_DISPATCH(ib, lb, CALL);
#undef CALL
  if (wide) {
    const size_t smem = (size_t)WARPS_PER_BLOCK * subtree_warp_words(v.n_classes) * sizeof(uint32_t);
#define CALL(I, L)                                                                                      \
  k_subtree_wide<I, L, Q><<<grid_for(k_subtree_wide<I, L, Q>, items, smem, persistent), THREADS_PER_BLOCK, smem, st>>>( \
      v, small, s, tv, cap_small)
    CT_DISPATCH(ib, lb, CALL);
#undef CALL
  }
  pf->end();
  pf->launched(CT_K_SUBTREE, wide ? 2 : 1);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int launch_reset_step(const LevelScratch& s, uint32_t n_nodes, const StepLists& lists, cudaStream_t st) {
  k_reset_step<<<1, 1, 0, st>>>(s.ctr, n_nodes, s.step, lists);
  current_prof()->launched(CT_K_CHILDREN);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

PartWork level_part_work(const View& v, const LevelScratch& s) {
  PartWork w;
  w.small = s.small_segs;
  w.n_small = &s.ctr->n_small_segs;
  w.cap_small = s.cap_nodes;
  w.big = s.big_segs;
  w.n_big = &s.ctr->n_big_segs;
  w.cap_big = s.cap_nodes;
  w.bchains = s.bchains;
  w.n_bchains = &s.ctr->n_bchains;
  w.cap_bchains = s.cap_bchains;
  w.huge = s.huge_segs;
  w.hchains = s.hchains;
  w.n_hchains = &s.ctr->n_hchains;
  w.cap_hchains = s.cap_hchains;
  w.ticket_huge = &s.ctr->ticket_huge;
  w.bit_words = v.bit_words;
  w.shape = s.part_shape;
  w.tiles = s.tiles;
  w.n_tiles = &s.ctr->n_tiles;
  w.cap_tiles = s.cap_status;
  w.status = s.status;
  w.cap_status = s.cap_status;
  w.ticket = &s.ctr->ticket;
  w.error = &s.ctr->error;
  w.n_features = v.n_features;
  return w;
}

namespace {
// Feature flags over a (row chunk, feature) grid: the minimum and maximum of
// each feature (as order-preserving bits, -0.0 folded onto +0.0), then
// whether some row holds a third value.
constexpr uint32_t FLAG_ROWS = 8192;  // rows per block

__global__ void k_ff_minmax(const float* __restrict__ x_fm, uint32_t n_rows, uint2* __restrict__ mm) {
  const uint32_t f = blockIdx.y;
  const float* xr = x_fm + (size_t)f * n_rows;
  const uint32_t lo = blockIdx.x * FLAG_ROWS, hi = min(lo + FLAG_ROWS, n_rows);
  uint32_t mn = 0xffffffffu, mx = 0u;
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const uint32_t o = f32_order(xr[i]);
    mn = min(mn, o);
    mx = max(mx, o);
  }
  mn = __reduce_min_sync(FULL, mn);
  mx = __reduce_max_sync(FULL, mx);
  if (lane_id() == 0) {
    atomicMin(&mm[f].x, mn);
    atomicMax(&mm[f].y, mx);
  }
}

__global__ void k_ff_third(const float* __restrict__ x_fm, uint32_t n_rows, const uint2* __restrict__ mm,
                           uint32_t* __restrict__ third) {
  const uint32_t f = blockIdx.y;
  const float* xr = x_fm + (size_t)f * n_rows;
  const uint32_t lo = blockIdx.x * FLAG_ROWS, hi = min(lo + FLAG_ROWS, n_rows);
  const uint2 b = mm[f];
  bool other = false;
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const uint32_t o = f32_order(xr[i]);
    other |= o != b.x && o != b.y;
  }
  if (__any_sync(FULL, other) && lane_id() == 0) atomicOr(third + (f >> 5), 1u << (f & 31));
}

__global__ void k_ff_final(const uint2* __restrict__ mm, const uint32_t* __restrict__ third, uint32_t n_features,
                           uint32_t* __restrict__ bits, float2* vals) {
  for (uint32_t f = threadIdx.x; f < n_features; f += blockDim.x) {
    if (vals) vals[f] = make_float2(f32_unorder(mm[f].x), f32_unorder(mm[f].y));
    if (!((third[f >> 5] >> (f & 31)) & 1u)) atomicOr(bits + (f >> 5), 1u << (f & 31));
  }
}
}  // namespace

// work: feature_flags_work_bytes(n_features) of device scratch (the
// per-feature minimum/maximum bits and the third-value words).
int feature_flags(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t* bits, float2* vals,
                  void* work, cudaStream_t st) {
  const uint32_t words = (n_features + 31) / 32;
  uint2* mm = reinterpret_cast<uint2*>(work);
  uint32_t* third = reinterpret_cast<uint32_t*>(mm + n_features);
  CT_CUDA_TRY(cudaMemsetAsync(bits, 0, words * sizeof(uint32_t), st));
  CT_CUDA_TRY(cudaMemsetAsync(third, 0, words * sizeof(uint32_t), st));
  CT_CUDA_TRY(cudaMemsetAsync(mm, 0xff, n_features * sizeof(uint2), st));  // min: all ones
  CT_CUDA_TRY(cudaMemset2DAsync(reinterpret_cast<char*>(mm) + 4, sizeof(uint2), 0, 4, n_features, st));  // max: 0
  const dim3 grid(ceil_div(n_rows, FLAG_ROWS), n_features);
  k_ff_minmax<<<grid, 256, 0, st>>>(x_fm, n_rows, mm);
  k_ff_third<<<grid, 256, 0, st>>>(x_fm, n_rows, mm, third);
  k_ff_final<<<1, 256, 0, st>>>(mm, third, n_features, bits, vals);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

size_t feature_flags_work_bytes(uint32_t n_features) {
  return n_features * sizeof(uint2) + ((n_features + 31) / 32) * sizeof(uint32_t);
}

namespace {
// Value bits of the virtual features: bit f of out[row] when x[f][row] is the
// feature's high value.
__global__ void k_vrow(const float* __restrict__ x_fm, uint32_t n_rows, uint64_t vmask, const float2* __restrict__ vval,
                       uint64_t* __restrict__ out) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
    uint64_t b = 0;
    for (uint64_t vm = vmask; vm; vm &= vm - 1) {
      const uint32_t f = (uint32_t)__ffsll((long long)vm) - 1;
      if (x_fm[(size_t)f * n_rows + r] == vval[f].y) b |= 1ull << f;
    }
    out[r] = b;
  }
}
}  // namespace

int virtual_rows(const float* x_fm, uint32_t n_rows, uint64_t vmask, const float2* vval, uint64_t* out,
                 cudaStream_t st) {
  k_vrow<<<std::min<uint32_t>(ceil_div(n_rows, 256), 148 * 8), 256, 0, st>>>(x_fm, n_rows, vmask, vval, out);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

Prof* current_prof() {
  static thread_local Prof prof;
  return &prof;
}

View make_view(const ct_problem* p, const ct_lists* l) {
  View v;
  v.x_fm = p->x_fm;
  v.labels = p->labels;
  v.si0 = l ? l->si0 : nullptr;
  v.si1 = l ? l->si1 : nullptr;
  v.mark = l ? l->mark : nullptr;
  v.n_slots = l ? l->n_slots : 0;
  v.bit_words = mark_bit_words(p->n_rows);
  v.bits = l && l->mark ? reinterpret_cast<uint32_t*>(l->mark + mark_bits_offset(p->n_rows, l->n_slots)) : nullptr;
  v.stride = l ? l->stride : 0;
  v.n_rows = p->n_rows;
  v.n_features = p->n_features;
  v.n_classes = p->n_classes;
  v.max_features = p->max_features;
  v.mss = p->min_samples_split;
  v.feistel_h = feistel_half_bits(p->n_features);
  v.row_mask = 0xffffffffu;
  v.lab_shift = 0;
  v.fbin = nullptr;
  v.vmask = 0;
  v.vrow = nullptr;
  v.vval = nullptr;
  v.vslot = 0;
  v.jobs = nullptr;
  v.slot_job = nullptr;
  v.slot_base = 0;
  v.sel_stride = p->max_features;
  v.mask_stride = mask_words(p->n_features);
  return v;
}

uint32_t fit_label_shift(const ct_problem* p) {
  const uint32_t row_bits = p->n_rows > 1 ? 32u - (uint32_t)__builtin_clz(p->n_rows - 1) : 1u;
  const uint32_t lab_bits = p->n_classes > 1 ? 32u - (uint32_t)__builtin_clz(p->n_classes - 1) : 0u;
  return (row_bits <= 31 && row_bits + lab_bits <= 8 * p->index_bytes) ? row_bits : 0u;
}

int check_problem(const ct_problem* p) {
  CT_ARG_CHECK(p != nullptr, "problem is NULL");
  CT_ARG_CHECK(p->x_fm && p->labels, "problem samples/labels are NULL");
  CT_ARG_CHECK(p->n_rows >= 1, "n_rows must be >= 1");
  CT_ARG_CHECK(p->n_features >= 1 && p->n_features <= CT_MAX_FEATURES, "n_features out of range");
  CT_ARG_CHECK(p->n_classes >= 1 && p->n_classes <= CT_MAX_CLASSES, "n_classes out of range");
  CT_ARG_CHECK(p->index_bytes == 2 || p->index_bytes == 4, "index_bytes must be 2 or 4");
  CT_ARG_CHECK(p->index_bytes == 4 || p->n_rows <= 0xFFFFu, "uint16 indices need n_rows <= 65535");
  CT_ARG_CHECK(p->label_bytes == 1 || p->label_bytes == 2, "label_bytes must be 1 or 2");
  CT_ARG_CHECK(p->label_bytes == 2 || p->n_classes <= 0xFFu, "uint8 labels need n_classes <= 255");
  CT_ARG_CHECK(p->max_features >= 1 && p->max_features <= p->n_features,
               "max_features must be in [1, n_features]");
  CT_ARG_CHECK(p->min_samples_split >= 1, "min_samples_split must be >= 1");
  return CT_OK;
}

}  // namespace ct
