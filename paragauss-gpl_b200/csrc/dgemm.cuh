// dgemm.cuh -- FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) tile engine.
//
// The FP64 path has no tcgen05 form (tcgen05.mma has no f64 kind), so the
// two dense contractions of the drop-in path run on the FP64 tensor pipe
// through warp-level mma.sync.  One CTA computes a 64x64 tile with 4 warps
// (32x32 each), K staged through shared memory in 16-deep slabs by cp.async
// with a NSTAGE-deep ring.
//
// Operand layouts (doubles):
//   MNC: element (k, mn) at base[k*ld + mn]   (mn contiguous)
//   KC : element (mn, k) at base[mn*ld + k]   (k contiguous)
// Callers pad every buffer so that tiles never leave the allocation: M, N to
// multiples of 64, K to multiples of 16, ld even (16-byte rows for cp.async).
#pragma once

#include <cstdint>

namespace pgxc {

constexpr int kBM = 64, kBN = 64, kBK = 16, kStages = 3;
constexpr int kPadMN = 4;   // MNC rows: 68 doubles (== 4 mod 16: conflict-free fragments)
constexpr int kPadK = 4;    // KC rows: 20 doubles
constexpr int kGemmThreads = 128;

template <bool KC, int BMN>
struct OpTile {
  // doubles per stage
  static constexpr int kElems = KC ? BMN * (kBK + kPadK) : kBK * (BMN + kPadMN);
  __device__ static __forceinline__ int idx(int mn, int k) {
    return KC ? mn * (kBK + kPadK) + k : k * (BMN + kPadMN) + mn;
  }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Load one K-slab [k0, k0+16) of a 64-wide operand tile at mn0 into smem.
template <bool KC>
__device__ __forceinline__ void load_slab(double* s, const double* __restrict__ g, int64_t ld, int64_t mn0,
                                          int64_t k0) {
  const int t = threadIdx.x;
  // 64*16 doubles = 512 16-byte chunks, 4 per thread
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int c = t + i * kGemmThreads;
    if (KC) {
      const int mn = c >> 3, k = (c & 7) * 2;
      cp_async16(s + OpTile<true, 64>::idx(mn, k), g + (mn0 + mn) * ld + k0 + k);
    } else {
      const int k = c >> 5, mn = (c & 31) * 2;
      cp_async16(s + OpTile<false, 64>::idx(mn, k), g + (k0 + k) * ld + mn0 + mn);
    }
  }
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// acc[mi][ni][e]: row = wm0 + mi*8 + lane/4, col = wn0 + ni*8 + 2*(lane%4) + e
struct Acc {
  double v[4][4][2];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) v[i][j][0] = v[i][j][1] = 0.0;
  }
};

// acc += A(m0:m0+64, k) * B(k, n0:n0+64) over k in [k_begin, k_end).
// smem must hold kStages * (OpTile<A_KC>::kElems + OpTile<B_KC>::kElems) doubles.
template <bool A_KC, bool B_KC>
__device__ __forceinline__ void gemm_tile(Acc& acc, const double* __restrict__ A, int64_t lda, int64_t m0,
                                          const double* __restrict__ B, int64_t ldb, int64_t n0, int64_t k_begin,
                                          int64_t k_end, double* smem) {
  constexpr int EA = OpTile<A_KC, 64>::kElems, EB = OpTile<B_KC, 64>::kElems;
  double* sA = smem;
  double* sB = smem + kStages * EA;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp >> 1) * 32, wn0 = (warp & 1) * 32;
  const int fr = lane >> 2, fk = lane & 3;
  const int nslab = (int)((k_end - k_begin) / kBK);
  // prologue
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nslab) {
      load_slab<A_KC>(sA + s * EA, A, lda, m0, k_begin + (int64_t)s * kBK);
      load_slab<B_KC>(sB + s * EB, B, ldb, n0, k_begin + (int64_t)s * kBK);
    }
    cp_async_commit();
  }
  for (int it = 0; it < nslab; ++it) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    // prefetch slab it + kStages - 1 into the stage consumed at it - 1
    {
      const int nx = it + kStages - 1;
      if (nx < nslab) {
        const int st = nx % kStages;
        load_slab<A_KC>(sA + st * EA, A, lda, m0, k_begin + (int64_t)nx * kBK);
        load_slab<B_KC>(sB + st * EB, B, ldb, n0, k_begin + (int64_t)nx * kBK);
      }
      cp_async_commit();
    }
    const double* a_s = sA + (it % kStages) * EA;
    const double* b_s = sB + (it % kStages) * EB;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = a_s[OpTile<A_KC, 64>::idx(wm0 + i * 8 + fr, kk + fk)];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = b_s[OpTile<B_KC, 64>::idx(wn0 + j * 8 + fr, kk + fk)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc.v[i][j], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

template <bool A_KC, bool B_KC>
constexpr int gemm_smem_bytes() {
  return kStages * (OpTile<A_KC, 64>::kElems + OpTile<B_KC, 64>::kElems) * (int)sizeof(double);
}

}  // namespace pgxc
