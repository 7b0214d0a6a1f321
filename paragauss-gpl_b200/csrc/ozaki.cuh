// ozaki.cuh -- the integer split ("Ozaki scheme") shared by the INT8
// tensor-core kernels.
//
// An FP64 operand row with power-of-two scale 2^e is rounded to the integer
// q = round(v 2^(34-e)) (|q| <= 2^34) and written as 5 balanced base-128
// digits d_0..d_4 (|d_s| <= 64), v ~= 2^e sum_s d_s 2^(-6-7s).  A product
// of two such operands keeps the digit pairs (s, t) with s + t <= 4 (15 INT8
// MMAs); the pairs of one group g = s + t share an INT32 accumulator D_g,
// which is exact (|d_s d_t| <= 2^12, K * 3 * 2^12 < 2^31 for K < 2^17).
// The accumulators are combined exactly in 64-bit integers,
//   x = sum_g D_g 2^(7(4-g)),  product = 2^(e_a + e_b - 40) x,
// and converted to FP64 once.  Truncation of the dropped pairs (s + t >= 5)
// and the rounding of q bound the relative error per product term by about
// 2^-34 of the operands' scales.
#pragma once

#include <cstdint>

#include "tc.cuh"

namespace pgxc {
namespace {

constexpr int kSlices = 5;  // 7-bit digits per operand
constexpr int kGroups = 5;  // digit-pair groups s + t = 0..4
constexpr int kPairs = 15;

// digit-pair list (s, t, group s + t); the first pair of each group starts its accumulator
__constant__ int c_oz_pairs[kPairs][3] = {{0, 0, 0}, {0, 1, 1}, {1, 0, 1}, {0, 2, 2}, {1, 1, 2},
                                          {2, 0, 2}, {0, 3, 3}, {1, 2, 3}, {2, 1, 3}, {3, 0, 3},
                                          {0, 4, 4}, {1, 3, 4}, {2, 2, 4}, {3, 1, 4}, {4, 0, 4}};
__host__ __device__ constexpr bool pair_leads(int q) { return q == 0 || q == 1 || q == 3 || q == 6 || q == 10; }

// offset of element (row r, K byte k) inside a rows x 32 K-major int8 block:
// core matrices of 8 rows x 16 bytes; LBO (K halves) = 128 B, SBO (8-row groups) = 256 B
__host__ __device__ constexpr int blk_off(int r, int k) {
  return (r & 7) * 16 + (k & 15) + (k >> 4) * 128 + (r >> 3) * 256;
}

// power-of-two exponent e with |v| / 2^e < 1 for all |v| <= mx (0 for mx == 0)
__device__ __forceinline__ int scale_exp(double mx) { return mx > 0.0 ? ilogb(mx) + 1 : 0; }

// 2^e built from the bit pattern, e clamped to the normal range [-1022, 1023]
// (clamping only touches operands or terms below 2^-960 in magnitude)
__device__ __forceinline__ double pow2(int e) {
  return __longlong_as_double((long long)(min(max(e, -1022), 1023) + 1023) << 52);
}
constexpr int kCombShift = -12 - 7 * (kGroups - 1);  // x * 2^kCombShift = sum_g 2^(-12-7g) D_g

// the integer q = round(v 2^(34-e)) of the split (|v| < 2^e)
__device__ __forceinline__ long long oz_int(double v, int e) { return __double2ll_rn(v * pow2(34 - e)); }

// 5 balanced base-128 digits of q, most significant first
__device__ __forceinline__ void oz_digits(long long q, int8_t (&d)[kSlices]) {
#pragma unroll
  for (int s = kSlices - 1; s >= 1; --s) {
    const long long r = ((q + 64) & 127) - 64;
    d[s] = (int8_t)r;
    q = (q - r) >> 7;
  }
  d[0] = (int8_t)q;  // |q| <= 64
}
__device__ __forceinline__ void digits(double v, int e, int8_t (&d)[kSlices]) { oz_digits(oz_int(v, e), d); }

// q + kOzOff has the base-128 digits u_s = d_s + 64 (u_0 in [0, 128], the
// others in [0, 127]): the balanced digits without carries
constexpr long long kOzOff = 64LL * ((1LL << 28) + (1LL << 21) + (1LL << 14) + (1LL << 7) + 1);

// the digits of four integers, one 32-bit word per slice (byte u = digit of q[u])
__device__ __forceinline__ void oz_pack4(const long long (&q)[4], uint32_t (&w)[kSlices]) {
  uint32_t u[4][kSlices];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long v = q[i] + kOzOff;
    const uint32_t lo = (uint32_t)v;
    u[i][0] = (uint32_t)(v >> 28);
    u[i][1] = (lo >> 21) & 127u;
    u[i][2] = (lo >> 14) & 127u;
    u[i][3] = (lo >> 7) & 127u;
    u[i][4] = lo & 127u;
  }
  // byte-wise u - 64 (mod 256) without carries between bytes: add 0xC0 to the
  // low 7 bits and fix bit 7 by XOR (u_0 = 128 gives 64)
#pragma unroll
  for (int s = 0; s < kSlices; ++s) {
    const uint32_t a = u[0][s] | (u[1][s] << 8) | (u[2][s] << 16) | (u[3][s] << 24);
    w[s] = ((a & 0x7f7f7f7fu) + 0x40404040u) ^ ((a & 0x80808080u) ^ 0x80808080u);
  }
}

// combine the kGroups INT32 accumulator values of one element (as loaded
// from TMEM) exactly into x = sum_g D_g 2^(7(4-g))
__device__ __forceinline__ double oz_combine(const uint32_t (&g)[kGroups]) {
  long long acc = 0;
#pragma unroll
  for (int i = 0; i < kGroups; ++i) acc += (long long)(int)g[i] << (7 * (kGroups - 1 - i));
  return (double)acc;
}

// issue the 15 digit-pair MMAs of one K step: A and B blocks of kSlices
// slices each (slice stride a_slice / b_slice bytes), accumulators at
// d_tmem + g * d_group columns
// (8-row groups of each slice a_sbo / b_sbo bytes apart)
__device__ __forceinline__ void oz_mma_pairs(uint32_t d_tmem, uint32_t d_group, uint32_t abase, uint32_t a_slice,
                                             uint32_t bbase, uint32_t b_slice, uint32_t idesc, bool first,
                                             uint32_t a_sbo = 256, uint32_t b_sbo = 256) {
#pragma unroll
  for (int q = 0; q < kPairs; ++q) {
    const int s = c_oz_pairs[q][0], t = c_oz_pairs[q][1], g = c_oz_pairs[q][2];
    const uint64_t ad = tc::smem_desc(abase + s * a_slice, 128, a_sbo);
    const uint64_t bd = tc::smem_desc(bbase + t * b_slice, 128, b_sbo);
    tc::mma_s8(d_tmem + g * d_group, ad, bd, idesc, !(first && pair_leads(q)));
  }
}

// The same 15 products as 5 MMAs: for digit slice s of A, the pairs (s, t),
// t = 0..4-s, go to the accumulator groups s + t, which are consecutive
// 48-column blocks of TMEM; with the 5 slices of B stored one after another
// (48 rows each, canonical layout) they are one MMA of N = 48 (5 - s) whose
// output starts at group s.  A is read from shared memory 5 times per K step
// instead of 15 (the MMAs are bound by shared-memory bandwidth otherwise).
// The first MMA (s = 0, N = 240) covers every group, so it alone starts the
// accumulators.
template <int NB>
__device__ __forceinline__ void oz_mma_fused(uint32_t d_tmem, uint32_t abase, uint32_t a_slice, uint32_t a_sbo,
                                             uint32_t bbase, bool first) {
#pragma unroll
  for (int s = 0; s < kSlices; ++s) {
    const uint64_t ad = tc::smem_desc(abase + s * a_slice, 128, a_sbo);
    const uint64_t bd = tc::smem_desc(bbase, 128, 256);
    tc::mma_s8(d_tmem + s * NB, ad, bd, tc::idesc_s8(128, NB * (kSlices - s)), !(first && s == 0));
  }
}

// Slice-interleaved K-major block: 8-row groups of [slice][8 rows x 32 bytes]
// (256 bytes per slice, 1280 per group), so that any run of whole 8-row
// groups is one contiguous range holding all 5 slices.  Within a slice the
// layout is the canonical one (LBO 128 between K halves, SBO 1280 between
// 8-row groups).
constexpr int kIlvGroup = kSlices * 256;
__host__ __device__ constexpr int ilv_off(int r, int k, int s) {
  return (r >> 3) * kIlvGroup + s * 256 + (r & 7) * 16 + (k & 15) + (k >> 4) * 128;
}

}  // namespace
}  // namespace pgxc
