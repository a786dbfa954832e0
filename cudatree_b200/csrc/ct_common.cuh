// Shared device/host definitions for the cudatree_b200 kernels.
//
// The split rule, the RNG streams and the feature permutation defined here are
// the canonical rule that the CPU oracle restates; every kernel that grows a
// tree (per-node form, level-synchronous form, warp subtrees) calls these so
// that all forms produce the same trees bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cudatree_b200.h"

namespace ct {

constexpr unsigned FULL = 0xffffffffu;
constexpr double DIFF_THRESHOLD = 0.00001;  // reference common_func.cu:1

// ---------------------------------------------------------------------------
// Counter-based RNG: SplitMix64 output function (Steele, Lea, Flood 2014).
// ---------------------------------------------------------------------------
constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;
constexpr uint64_t K_TREE = 0x243F6A8885A308D3ull;
constexpr uint64_t K_BOOT = 0x6A09E667F3BCC909ull;
constexpr uint64_t K_ROOT = 0xBB67AE8584CAA73Bull;
constexpr uint64_t K_LEFT = 0xA54FF53A5F1D36F1ull;
constexpr uint64_t K_RIGHT = 0x3C6EF372FE94F82Bull;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t tree_key(uint64_t seed, uint32_t tree) {
  return mix64(mix64(seed ^ K_TREE) + (uint64_t)(tree + 1) * GOLDEN);
}
__host__ __device__ __forceinline__ uint64_t root_key(uint64_t tkey) { return mix64(tkey ^ K_ROOT); }
__host__ __device__ __forceinline__ uint64_t child_key(uint64_t key, int side) {
  return mix64(key ^ (side ? K_RIGHT : K_LEFT));
}
__host__ __device__ __forceinline__ uint64_t boot_key(uint64_t tkey) { return mix64(tkey ^ K_BOOT); }
// i-th bootstrap draw in [0, n): (hi32(splitmix(bk, i)) * n) >> 32
__host__ __device__ __forceinline__ uint32_t boot_draw(uint64_t bk, uint64_t i, uint32_t n) {
  uint64_t u = mix64(bk + (i + 1) * GOLDEN);
  return (uint32_t)(((u >> 32) * (uint64_t)n) >> 32);
}

// Keyed 4-round Feistel permutation of [0, 4^h), cycle-walked onto [0, F).
__host__ __device__ __forceinline__ int feistel_half_bits(uint32_t n_features) {
  uint32_t v = n_features - 1;
  int bits = 0;
  while (v) { ++bits; v >>= 1; }
  int h = (bits + 1) / 2;
  return h < 1 ? 1 : h;
}
__host__ __device__ __forceinline__ uint32_t feistel(uint32_t x, uint64_t key, int h) {
  const uint32_t mask = (1u << h) - 1u;
  uint32_t l = x >> h, r = x & mask;
#pragma unroll
  for (int round = 0; round < 4; ++round) {
    uint32_t fr = (uint32_t)(mix64(key + (uint64_t)(((uint32_t)round << 16) | r) * GOLDEN) & mask);
    uint32_t nl = r;
    r = l ^ fr;
    l = nl;
  }
  return (l << h) | r;
}
__host__ __device__ __forceinline__ uint32_t feature_perm(uint32_t i, uint32_t n_features, uint64_t key, int h) {
  uint32_t x = feistel(i, key, h);
  // Terminates: the cycle of the permutation through i returns to i < F.
  while (x >= n_features) x = feistel(x, key, h);
  return x;
}

// ---------------------------------------------------------------------------
// Float ordering: -0.0 folded onto +0.0, monotone uint32 image.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t f32_order(float x) {
  uint32_t b = __float_as_uint(__fadd_rn(x, 0.0f));
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float f32_unorder(uint32_t k) {
  uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(b);
}

// ---------------------------------------------------------------------------
// Split arithmetic (reference dfs_module.cu:400-407), no contraction.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool is_candidate(float x, float x_next) {
  return __dadd_rn((double)x, DIFF_THRESHOLD) < (double)x_next;
}
// is_candidate for sorted neighbours (x <= x_next) with the double test only
// where it can matter: equal values never qualify, and a float gap above 1e-4
// (true gap > 9.99e-5 after the subtraction's 2^-24 relative rounding) always
// does, since the double sum x + 1e-5 exceeds x by less than that.
__device__ __forceinline__ bool is_candidate_sorted(float x, float x_next) {
  if (!(x_next > x)) return false;
  if (x_next - x > 1e-4f) return true;
  return is_candidate(x, x_next);
}
__device__ __forceinline__ double gini_part(int64_t sq_sum, double n_side, double n_total) {
  double ratio = __ddiv_rn((double)sq_sum, __dmul_rn(n_side, n_side));
  return __dmul_rn(__dsub_rn(1.0, ratio), __ddiv_rn(n_side, n_total));
}
__device__ __forceinline__ float midpoint(float a, float b) {
  return __double2float_rn(__dmul_rn(__dadd_rn((double)a, (double)b), 0.5));
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ int64_t warp_incl_scan_i64(int64_t v) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    int64_t o = __shfl_up_sync(FULL, v, s);
    if (lane >= (unsigned)s) v += o;
  }
  return v;
}
__device__ __forceinline__ int32_t warp_incl_scan_i32(int32_t v) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const int32_t o = __shfl_up_sync(FULL, v, s);
    if (lane >= (unsigned)s) v += o;
  }
  return v;
}
__device__ __forceinline__ int64_t warp_sum_i64(int64_t v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(FULL, v, s);
  return v;
}
__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(FULL, v, s);
  return v;
}

// Lexicographic (score, a, b) minimum across the warp; result in every lane.
__device__ __forceinline__ void warp_argmin3(double& score, uint32_t& a, uint32_t& b, float& p, float& q) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    double os = __shfl_xor_sync(FULL, score, s);
    uint32_t oa = __shfl_xor_sync(FULL, a, s);
    uint32_t ob = __shfl_xor_sync(FULL, b, s);
    float op = __shfl_xor_sync(FULL, p, s);
    float oq = __shfl_xor_sync(FULL, q, s);
    bool take = (os < score) || (os == score && (oa < a || (oa == a && ob < b)));
    if (take) { score = os; a = oa; b = ob; p = op; q = oq; }
  }
}

template <typename T>
__device__ __forceinline__ T ld_idx(const void* base, size_t i) {
  return reinterpret_cast<const T*>(base)[i];
}

__host__ __device__ __forceinline__ uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace ct
