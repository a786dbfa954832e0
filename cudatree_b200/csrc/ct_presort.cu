// Stable per-feature presort on the device (replaces the host
// np.argsort of random_forest.py:247).
//
// Keys are the order-preserving uint32 image of each float (with -0.0 folded
// onto +0.0); values are row ids.  Four 8-bit LSD radix passes, each
//   k_digit_hist  per (tile, feature) digit histogram,
//   k_digit_scan  per feature exclusive scan over (digit, tile),
//   k_digit_move  stable scatter: warp-level ranks from __match_any_sync,
//                 then per-digit prefix over the tile's warps.
// A stable sort of keys that start in row order gives ties in row order,
// which is the tie rule the split search and the leaf labels rely on.
// Features with at most two distinct keys (one-hot and other binary columns;
// feature_flags finds them) take one pass instead of four: the same three
// kernels with the digit "key is the feature's larger key", a stable
// partition of the rows in row order.  Each kernel's blocks of the other kind
// of feature return at once.
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr int RS_WARPS = 8;
constexpr int RS_ROUNDS = 16;
constexpr uint32_t RS_TILE = RS_WARPS * RS_ROUNDS * 32;  // 4096
constexpr int RS_THREADS = RS_WARPS * 32;

struct RadixArgs {
  const float* x;          // pass 0 source
  const uint32_t* kin;
  const uint32_t* vin;
  uint32_t* kout;
  uint32_t* vout;
  void* final_out;         // last pass: row ids, index_bytes wide
  uint32_t* hist;          // [F][256][tiles]
  uint32_t n;
  uint32_t tiles;
  uint32_t shift;
  uint32_t first;
  uint32_t last;
  uint32_t index_bytes;
  uint32_t tv_pass;        // 1: the pass of the two-valued features; 0: a radix pass of the others
  const uint32_t* two;     // bit f: feature f has at most two distinct keys
  const uint2* mm;         // per feature: its (smallest, largest) key
};

__device__ __forceinline__ bool skip_feature(const RadixArgs& a, uint32_t f) {
  const bool tv = (a.two[f >> 5] >> (f & 31)) & 1u;
  return tv != (a.tv_pass != 0);
}
__device__ __forceinline__ uint32_t digit(const RadixArgs& a, uint32_t f, uint32_t key) {
  return a.tv_pass ? (key == a.mm[f].y ? 1u : 0u) : (key >> a.shift) & 255u;
}

__device__ __forceinline__ uint32_t load_key(const RadixArgs& a, uint32_t f, uint32_t i) {
  return a.first ? f32_order(a.x[(size_t)f * a.n + i]) : a.kin[(size_t)f * a.n + i];
}

__global__ void __launch_bounds__(RS_THREADS) k_digit_hist(RadixArgs a) {
  __shared__ uint32_t h[256];
  const uint32_t tile = blockIdx.x, f = blockIdx.y;
  if (skip_feature(a, f)) return;
  for (uint32_t d = threadIdx.x; d < 256; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const uint32_t lo = tile * RS_TILE, hi = min(lo + RS_TILE, a.n);
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    atomicAdd(&h[digit(a, f, load_key(a, f, i))], 1u);
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < 256; d += blockDim.x)
    a.hist[((size_t)f * 256 + d) * a.tiles + tile] = h[d];
}

__global__ void __launch_bounds__(1024) k_digit_scan(RadixArgs a) {
  __shared__ uint32_t warp_tot[32];
  const uint32_t f = blockIdx.x, tiles = a.tiles;
  if (skip_feature(a, f)) return;
  uint32_t* row = a.hist + (size_t)f * 256 * tiles;
  const uint32_t L = 256 * tiles;
  const uint32_t per = (L + blockDim.x - 1) / blockDim.x;
  const uint32_t lo = min(threadIdx.x * per, L), hi = min(lo + per, L);
  uint32_t sum = 0;
  for (uint32_t i = lo; i < hi; ++i) sum += row[i];
  // block exclusive scan of per-thread sums
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = sum;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const uint32_t o = __shfl_up_sync(FULL, inc, s);
    if (lane >= (uint32_t)s) inc += o;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const uint32_t o = __shfl_up_sync(FULL, t, s);
      if (lane >= (uint32_t)s) t += o;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  uint32_t run = inc - sum + (warp ? warp_tot[warp - 1] : 0);
  for (uint32_t i = lo; i < hi; ++i) {
    const uint32_t v = row[i];
    row[i] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(RS_THREADS) k_digit_move(RadixArgs a) {
  __shared__ uint32_t wcnt[RS_WARPS][256];
  const uint32_t tile = blockIdx.x, f = blockIdx.y;
  if (skip_feature(a, f)) return;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t d = lane; d < 256; d += 32) wcnt[warp][d] = 0;
  __syncwarp();
  const uint32_t lo = tile * RS_TILE + warp * RS_ROUNDS * 32;
  uint32_t key[RS_ROUNDS], val[RS_ROUNDS], rank[RS_ROUNDS];
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    const uint32_t i = lo + r * 32 + lane;
    const bool ok = i < a.n;
    key[r] = ok ? load_key(a, f, i) : 0xffffffffu;
    val[r] = ok ? (a.first ? i : a.vin[(size_t)f * a.n + i]) : 0u;
    const uint32_t d = ok ? digit(a, f, key[r]) : 256u;
    const unsigned grp = __match_any_sync(FULL, d);
    rank[r] = ok ? wcnt[warp][d] + __popc(grp & lt) : 0u;
    __syncwarp();
    if (ok && (grp >> lane) == 1u) wcnt[warp][d] += __popc(grp);
    __syncwarp();
  }
  __syncthreads();
  // exclusive prefix over warps, per digit (in place)
  for (uint32_t d = threadIdx.x; d < 256; d += blockDim.x) {
    uint32_t run = a.hist[((size_t)f * 256 + d) * a.tiles + tile];
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
      const uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    const uint32_t i = lo + r * 32 + lane;
    if (i >= a.n) continue;
    const uint32_t d = digit(a, f, key[r]);
    const uint32_t dst = wcnt[warp][d] + rank[r];
    if (dst >= a.n) continue;
    if (a.last) {
      if (a.index_bytes == 2)
        reinterpret_cast<uint16_t*>(a.final_out)[(size_t)f * a.n + dst] = (uint16_t)val[r];
      else
        reinterpret_cast<uint32_t*>(a.final_out)[(size_t)f * a.n + dst] = val[r];
    } else {
      a.kout[(size_t)f * a.n + dst] = key[r];
      a.vout[(size_t)f * a.n + dst] = val[r];
    }
  }
}

}  // namespace

// Row-major [n_rows][n_cols] -> column-major [n_cols][n_rows] through a
// 32x33 shared-memory tile (coalesced reads and writes); row tiles are
// strided over gridDim.y.  A NaN anywhere sets *nan_flag (when given), so
// the input check needs no pass over x on the host.
__global__ void k_transpose(const float* __restrict__ in, uint32_t n_rows, uint32_t n_cols, float* __restrict__ out,
                            uint32_t* nan_flag) {
  __shared__ float tile[32][33];
  const uint32_t c0 = blockIdx.x * 32;
  bool nan = false;
  for (uint32_t r0 = blockIdx.y * 32; r0 < n_rows; r0 += gridDim.y * 32) {
    for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
      const uint32_t r = r0 + k, c = c0 + threadIdx.x;
      if (r < n_rows && c < n_cols) {
        const float v = in[(size_t)r * n_cols + c];
        nan |= v != v;
        tile[k][threadIdx.x] = v;
      }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
      const uint32_t c = c0 + k, r = r0 + threadIdx.x;
      if (r < n_rows && c < n_cols) out[(size_t)c * n_rows + r] = tile[threadIdx.x][k];
    }
    __syncthreads();
  }
  if (__syncthreads_or(nan) && threadIdx.x == 0 && threadIdx.y == 0 && nan_flag) atomicOr(nan_flag, 1u);
}

size_t presort_workspace_bytes(uint32_t n_rows, uint32_t n_features) {
  const size_t tiles = ceil_div(n_rows, RS_TILE);
  const size_t elems = (size_t)n_rows * n_features;
  return 4 * elems * sizeof(uint32_t) + (size_t)n_features * 256 * tiles * sizeof(uint32_t) +
         ((n_features + 31) / 32) * sizeof(uint32_t) + feature_flags_work_bytes(n_features) + 7 * 256;
}

int presort(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t index_bytes, void* out, void* ws,
            size_t wsb, cudaStream_t st) {
  CT_ARG_CHECK(x_fm && out && ws, "presort: NULL argument");
  CT_ARG_CHECK(n_rows >= 1 && n_features >= 1 && n_features <= 65535u, "presort: bad shape");
  CT_ARG_CHECK(index_bytes == 4 || (index_bytes == 2 && n_rows <= 0xFFFFu), "presort: bad index width");
  const uint32_t tiles = ceil_div(n_rows, RS_TILE);
  const size_t elems = (size_t)n_rows * n_features;
  Arena ar{reinterpret_cast<char*>(ws), wsb, 0};
  uint32_t* k0 = ar.take<uint32_t>(elems);
  uint32_t* v0 = ar.take<uint32_t>(elems);
  uint32_t* k1 = ar.take<uint32_t>(elems);
  uint32_t* v1 = ar.take<uint32_t>(elems);
  uint32_t* hist = ar.take<uint32_t>((size_t)n_features * 256 * tiles);
  uint32_t* two = ar.take<uint32_t>((n_features + 31) / 32);
  char* ffw = ar.take<char>(feature_flags_work_bytes(n_features));  // starts with the (min, max) keys
  if (!hist || !two || !ffw) {
    set_last_error("presort workspace too small");
    return CT_ERR_OOM;
  }
  RadixArgs a;
  a.x = x_fm;
  a.final_out = out;
  a.hist = hist;
  a.n = n_rows;
  a.tiles = tiles;
  a.index_bytes = index_bytes;
  CT_TRY(feature_flags(x_fm, n_rows, n_features, two, nullptr, ffw, st));
  a.two = two;
  a.mm = reinterpret_cast<const uint2*>(ffw);
  a.tv_pass = 0;
  const dim3 grid(tiles, n_features);
  for (uint32_t pass = 0; pass < 4; ++pass) {
    a.shift = pass * 8;
    a.first = pass == 0;
    a.last = pass == 3;
    a.kin = (pass & 1) ? k0 : k1;
    a.vin = (pass & 1) ? v0 : v1;
    a.kout = (pass & 1) ? k1 : k0;
    a.vout = (pass & 1) ? v1 : v0;
    k_digit_hist<<<grid, RS_THREADS, 0, st>>>(a);
    k_digit_scan<<<n_features, 1024, 0, st>>>(a);
    k_digit_move<<<grid, RS_THREADS, 0, st>>>(a);
  }
  // the two-valued features: one stable partition pass from x to the output
  a.tv_pass = 1;
  a.shift = 0;
  a.first = 1;
  a.last = 1;
  k_digit_hist<<<grid, RS_THREADS, 0, st>>>(a);
  k_digit_scan<<<n_features, 1024, 0, st>>>(a);
  k_digit_move<<<grid, RS_THREADS, 0, st>>>(a);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

int transpose_rows(const float* x_rm, uint32_t n_rows, uint32_t n_cols, float* x_cm, cudaStream_t st,
                   uint32_t* nan_flag) {
  CT_ARG_CHECK(x_rm && x_cm, "transpose: NULL argument");
  if (n_rows == 0 || n_cols == 0) return CT_OK;
  CT_ARG_CHECK(ceil_div(n_cols, 32) <= 0x7fffffffu, "transpose: too many columns");
  const dim3 grid(ceil_div(n_cols, 32), std::min<uint32_t>(ceil_div(n_rows, 32), 65535u));
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(x_rm, n_rows, n_cols, x_cm, nan_flag);
  CT_CUDA_TRY(cudaGetLastError());
  return CT_OK;
}

}  // namespace ct
