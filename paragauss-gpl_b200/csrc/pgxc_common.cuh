// pgxc_common.cuh -- shared device-side definitions of libpgxc.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pgxc.h"

namespace pgxc {

// Maximum angular momentum handled by the basis kernels (f functions).
constexpr int kMaxL = 3;
// Radial functions evaluated per pass of the basis kernel; shells with more
// radial functions are processed in several passes.
constexpr int kRadGroup = 8;

// One (atom, l) shell of the orbital basis, device copy.
struct DevShell {
  int atom;
  int l;
  int nexp;
  int nunc;
  int ncontr;
  int nrad;      // nunc + ncontr
  int exp_off;   // into exponents / norms
  int con_off;   // into contractions (nexp x ncontr column-major)
  int f0;        // first basis function
  int seg;       // 1: every contraction uses its own contiguous range of primitives
  int rad_off;   // into the radial-range table (seg shells): [lo, hi) per contraction
  int pad_;
  double min_exp;  // smallest exponent: bounds the shell's spatial extent
};

// Symmetry adaptation: independent function i of shell l is
// sum_m sa[l][i][m] Y_lm; identity when sa_identity is set.
struct DevSA {
  double c[kMaxL + 1][2 * kMaxL + 1][2 * kMaxL + 1];
  int identity;
};

// Tile size of the potential/density-matrix blocking (functions).
constexpr int kTile = 64;

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Thread count of a block rounded up to whole groups of four warps.  Every
// kernel of the library launches such blocks: a tensor-core CTA placed on an
// SM beside other CTAs then starts on a warp slot that is a multiple of four,
// so that its warp w sits in sub-partition w % 4, whose TMEM lanes
// 32 (w % 4) .. 32 (w % 4) + 31 its tcgen05.ld addresses.
__host__ __device__ constexpr int kBlock4(int threads) { return (threads + 127) / 128 * 128; }

// Raise, never lower, a kernel's dynamic shared-memory limit.  The limit
// belongs to the function, shared by every context of the process: a
// context whose tiles list fewer functions must not undercut the launches of
// another that are still queued or captured in a graph.
template <typename Kernel>
inline cudaError_t raise_smem_limit(Kernel kernel, int bytes) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if (fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace pgxc
