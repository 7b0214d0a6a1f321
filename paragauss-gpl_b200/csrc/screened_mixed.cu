// screened_mixed.cu -- INT8 tensor-core stages of the screened XC build.
//
// Both contractions of a tile run on tcgen05.mma kind::i8 with the Ozaki
// split of ozaki.cuh (15 digit-pair MMAs per K step, exact INT32
// accumulation in TMEM, FP64 combination):
//
//   k_sm_quant_pts   phi_t -> INT8 digits, one scale per point          (A of X)
//   k_sm_rowexp_P,   P -> packed digits P8[nu][mu] (5 bytes of a 64-bit
//   k_sm_quant_P     word), one scale per row nu                       (B of X)
//   k_sm_density     X = phi_t P[S_t, S_t], 128 points x 48 slots per MMA;
//                    A by bulk copy, B gathered from P8 by four producer
//                    warps, two TMEM accumulator sets (MMA of slot block j+1
//                    overlaps the epilogue of block j); fused FP64 epilogue
//                    rho += X phi, grad rho += 2 X grad phi
//   k_sm_zquant      Z = A phi (+ B . grad phi) in FP64 and the digits of Z
//                    and phi, one scale per (tile, slot)                (A, B of V)
//   k_sm_vpot        H[S_t, S_t] += Z_t^T phi_t, 128 x 48 slot blocks, K = the
//                    tile's 128 points; scaled in FP64 and scatter-added
//                    into the full matrix with atomics
//
// Every mbarrier wait is bounded (tc::kWaitLimit); a wait that runs out sets
// the device error flag and the kernel winds down.
#include <algorithm>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "ozaki.cuh"
#include "screened_mixed.h"
#include "tc.cuh"

namespace pgxc {

namespace {

constexpr int kM = 128;                    // MMA M (points in X, slots in V)
constexpr int kN = 48;                     // MMA N (slots)
constexpr int kBlkA = kM * 32;             // one slice of a 128-row x 32-byte K block
constexpr int kBlkB = kN * 32;             // one slice of a 48-row x 32-byte K block
constexpr int kOpA = kSlices * kBlkA;      // 20480
constexpr int kOpB = kSlices * kBlkB;      // 7680
constexpr int kAccCols = kGroups * kN;     // 240 TMEM columns per accumulator set
constexpr int kDStages = 3;                // density: A (phi digit) ring
constexpr int kBStages = 6;                // density: gathered B (P digit) ring
constexpr int kVStages = 6;
constexpr int kDigBytesPerSlot = 640;      // 128 points x 5 slices

}  // namespace

struct ScreenMixed {
  int64_t nbas = 0, ldc = 0;
  bool gga = false;
  int64_t chunk_slots = 0, chunk_tiles = 0;
  int max_n = 0;
  unsigned long long* P8 = nullptr;  // [nbas][nbas]
  int* e_P = nullptr;                // [nbas]
  int8_t* tA = nullptr;              // density A digits, [slot block of 32][slice][128 x 32] per tile
  int* e_pt = nullptr;               // [chunk_tiles * 128]
  int8_t* tZ = nullptr;              // V operand digits, [kstep][slice][n x 32] per tile
  int8_t* tF = nullptr;
  int* e_Z = nullptr;                // [chunk_slots]
  int* e_F = nullptr;
  int* err = nullptr;
  int nsm = 148;
  std::vector<void*> allocs;
};

namespace {

template <typename T>
cudaError_t sm_alloc(ScreenMixed* m, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) {
    m->allocs.push_back(q);
    *p = (T*)q;
  }
  return e;
}

// ---------------------------------------------------------------------------
// operands
// ---------------------------------------------------------------------------
__global__ void k_sm_rowexp_P(const double* __restrict__ P, int64_t ldc, int64_t nbas, int* __restrict__ e) {
  const double* row = P + (int64_t)blockIdx.x * ldc;
  double mx = 0.0;
  for (int64_t j = threadIdx.x; j < nbas; j += blockDim.x) mx = fmax(mx, fabs(row[j]));
  __shared__ double red[256];
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) e[blockIdx.x] = scale_exp(red[0]);
}

// P8[nu][mu]: byte s = digit s of P[nu][mu] at the row scale 2^e_P[nu]
__global__ void k_sm_quant_P(const double* __restrict__ P, int64_t ldc, int64_t nbas, const int* __restrict__ e_P,
                             unsigned long long* __restrict__ P8) {
  const int64_t total = nbas * nbas;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t nu = i / nbas, mu = i - nu * nbas;
    int8_t d[kSlices];
    digits(P[nu * ldc + mu], e_P[nu], d);
    unsigned long long w = 0;
#pragma unroll
    for (int s = 0; s < kSlices; ++s) w |= (unsigned long long)(uint8_t)d[s] << (8 * s);
    P8[i] = w;
  }
}

// rows = the tile's 128 points, K = its slots; one scale per point (largest
// |phi| over the tile's slots)
__global__ void __launch_bounds__(128) k_sm_quant_pts(const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
                                                      const double* __restrict__ phi, int* __restrict__ e_pt,
                                                      int8_t* __restrict__ tA) {
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int p = threadIdx.x;
  const double* src = phi + sb * 128 + p;
  double m8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; i += 8) {  // n is a multiple of 32
#pragma unroll
    for (int j = 0; j < 8; ++j) m8[j] = fmax(m8[j], fabs(src[(int64_t)(i + j) * 128]));
  }
  double mx = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) mx = fmax(mx, m8[j]);
  const int e = scale_exp(mx);
  e_pt[(int64_t)blockIdx.x * 128 + p] = e;
  int8_t* dst = tA + sb * kDigBytesPerSlot;
  for (int kb = 0; kb < n / 32; ++kb) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t w[4][kSlices];
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        long long q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = oz_int(src[(int64_t)(kb * 32 + h * 16 + g * 4 + u) * 128], e);
        oz_pack4(q, w[g]);
      }
#pragma unroll
      for (int s = 0; s < kSlices; ++s)
        *reinterpret_cast<uint4*>(dst + (int64_t)kb * kOpA + s * kBlkA + blk_off(p, h * 16)) =
            make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
    }
  }
}

// byte `sl` of each of 8 packed digit words -> one 64-bit row of 8 digits
__device__ __forceinline__ unsigned long long gather_slice(const unsigned long long (&w)[8], int sl) {
  uint32_t lo = 0, hi = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    lo |= ((uint32_t)(w[u] >> (8 * sl)) & 0xffu) << (8 * u);
    hi |= ((uint32_t)(w[u + 4] >> (8 * sl)) & 0xffu) << (8 * u);
  }
  return (unsigned long long)lo | ((unsigned long long)hi << 32);
}

// ---------------------------------------------------------------------------
// X = phi_t P[S_t, S_t] with fused rho / grad rho
// ---------------------------------------------------------------------------
// epilogue operands: phi (and grad phi) of 6 slots x 128 points per buffer
constexpr int kECols = 6;
constexpr int kERing = 4;
constexpr int kEBuf = 4 * kECols * 128;  // doubles
struct DensSmem {
  alignas(1024) int8_t a[kDStages][kOpA];
  alignas(1024) int8_t b[kBStages][kOpB];
  alignas(128) double e[kERing][kEBuf];   // [array][column][point]
  uint64_t full[kDStages];
  uint64_t empty[kDStages];
  uint64_t b_full[kBStages];
  uint64_t b_empty[kBStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t e_full[kERing];
  uint64_t e_empty[kERing];
  uint32_t tslot;
};
// warps 0-7 epilogue, 8 MMA, 9 A copies, 10-13 B gather, 14 epilogue-operand copies
constexpr int kDensThreads = 480;

// TMEM -> 16 + 8 combined FP64 values of one accumulator set (columns c0..c0+23)
__device__ __forceinline__ void read_acc24(uint32_t taddr, double (&x)[24]) {
  {
    uint32_t r[kGroups][16];
#pragma unroll
    for (int g = 0; g < kGroups; ++g) tc::tmem_ld16u(taddr + g * kN, r[g]);
    tc::tmem_ld_wait();
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      uint32_t v[kGroups];
#pragma unroll
      for (int g = 0; g < kGroups; ++g) v[g] = r[g][c];
      x[c] = oz_combine(v);
    }
  }
  {
    uint32_t r[kGroups][8];
#pragma unroll
    for (int g = 0; g < kGroups; ++g) tc::tmem_ld8(taddr + g * kN + 16, r[g]);
    tc::tmem_ld_wait();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint32_t v[kGroups];
#pragma unroll
      for (int g = 0; g < kGroups; ++g) v[g] = r[g][c];
      x[16 + c] = oz_combine(v);
    }
  }
}

// Persistent: CTA c takes the chunk's tiles c, c + G, c + 2G, ... (G = grid
// size); the copy / MMA / epilogue pipeline runs on across tile boundaries.
// rho and grad rho are accumulated with atomics (the two column halves of a
// point and nothing else), so they must be zero on entry.
template <bool GGA>
__global__ void __launch_bounds__(kDensThreads, 1)
    k_sm_density(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t nt,
                 int64_t s0, const int8_t* __restrict__ tA, const int* __restrict__ e_pt,
                 const unsigned long long* __restrict__ P8, const int* __restrict__ e_P, int64_t nbas,
                 const double* __restrict__ phi, const double* __restrict__ gx, const double* __restrict__ gy,
                 const double* __restrict__ gz, double* __restrict__ rho, double* __restrict__ grx,
                 double* __restrict__ gry, double* __restrict__ grz, int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  DensSmem& S = *reinterpret_cast<DensSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int s = 0; s < kDStages; ++s) {
      tc::mbar_init(&S.full[s], 1);
      tc::mbar_init(&S.empty[s], 1);
    }
    for (int s = 0; s < kBStages; ++s) {
      tc::mbar_init(&S.b_full[s], 128);
      tc::mbar_init(&S.b_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&S.acc_full[b], 1);
      tc::mbar_init(&S.acc_empty[b], 256);
    }
    for (int r = 0; r < kERing; ++r) {
      tc::mbar_init(&S.e_full[r], 1);
      tc::mbar_init(&S.e_empty[r], 128);
    }
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  bool ok = true;
  if (warp == 14) {
    if (lane == 0) {  // epilogue operands: per slot block j, half h, group u: 6 slots of phi (grad phi)
      int e = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nN = (n + kN - 1) / kN;
        for (int j = 0; j < nN && ok; ++j) {
          if (j + 1 < nN) {  // next block into L2
            const int rows = min(kN, n - (j + 1) * kN);
            const int64_t off = (sb + (int64_t)(j + 1) * kN) * 128;
            const uint32_t bytes = (uint32_t)rows * 128 * sizeof(double);
            tc::bulk_prefetch_l2(phi + off, bytes);
            if (GGA) {
              tc::bulk_prefetch_l2(gx + off, bytes);
              tc::bulk_prefetch_l2(gy + off, bytes);
              tc::bulk_prefetch_l2(gz + off, bytes);
            }
          }
          for (int u = 0; u < 4 && ok; ++u)
            for (int h = 0; h < 2; ++h, ++e) {
              const int r = e % kERing;
              if (e >= kERing && !tc::mbar_wait(&S.e_empty[r], ((e / kERing) - 1) & 1)) {
                ok = false;
                break;
              }
              const int c0 = j * kN + h * 24 + u * kECols;
              const int nc = max(0, min(kECols, n - c0));
              if (nc == 0) {
                tc::mbar_arrive(&S.e_full[r]);
                continue;
              }
              const uint32_t bytes = (uint32_t)nc * 128 * sizeof(double);
              const int64_t off = (sb + c0) * 128;
              tc::mbar_expect_tx(&S.e_full[r], (GGA ? 4 : 1) * bytes);
              tc::bulk_g2s(S.e[r], phi + off, bytes, &S.e_full[r]);
              if (GGA) {
                tc::bulk_g2s(S.e[r] + kECols * 128, gx + off, bytes, &S.e_full[r]);
                tc::bulk_g2s(S.e[r] + 2 * kECols * 128, gy + off, bytes, &S.e_full[r]);
                tc::bulk_g2s(S.e[r] + 3 * kECols * 128, gz + off, bytes, &S.e_full[r]);
              }
            }
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 8) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = tc::idesc_s8(kM, kN);
      int it = 0, jj = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nK = n / 32, nN = (n + kN - 1) / kN;
        for (int j = 0; j < nN && ok; ++j, ++jj) {
          const int b = jj & 1;
          if (jj >= 2 && !tc::mbar_wait(&S.acc_empty[b], ((jj >> 1) - 1) & 1)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          for (int k = 0; k < nK; ++k, ++it) {
            const int s = it % kDStages, sbb = it % kBStages;
            if (!tc::mbar_wait(&S.full[s], (it / kDStages) & 1) ||
                !tc::mbar_wait(&S.b_full[sbb], (it / kBStages) & 1)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
            oz_mma_pairs(tbase + b * kAccCols, kN, tc::smem_u32(S.a[s]), kBlkA, tc::smem_u32(S.b[sbb]), kBlkB, idesc,
                         k == 0);
            tc::mma_commit(&S.empty[s]);
            tc::mma_commit(&S.b_empty[sbb]);
          }
          tc::mma_commit(&S.acc_full[b]);
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 9) {
    if (lane == 0) {  // A producer: digits of phi, one 32-slot K block per stage
      int it = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nK = n / 32, nN = (n + kN - 1) / kN;
        const int8_t* src = tA + sb * kDigBytesPerSlot;
        for (int j = 0; j < nN && ok; ++j)
          for (int k = 0; k < nK; ++k, ++it) {
            const int s = it % kDStages;
            if (it >= kDStages && !tc::mbar_wait(&S.empty[s], ((it / kDStages) - 1) & 1)) {
              ok = false;
              break;
            }
            tc::mbar_expect_tx(&S.full[s], kOpA);
            tc::bulk_g2s(S.a[s], src + (int64_t)k * kOpA, kOpA, &S.full[s]);
          }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp >= 10 && warp < 14) {  // B producers: P8[fn(nu)][fn(mu)] gathered into the K-major digit block
    // thread g: tasks g and g + 128 (rows r = task / 4, 8 K values from 8 (task % 4));
    // warps 10-11 have two tasks, 12-13 one (uniform per warp)
    const int g = tid - 320;
    const bool two = g < kN * 4 - 128;
    int it = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
      const int64_t sg = tso[t0 + ti];
      const int n = (int)(tso[t0 + ti + 1] - sg);
      const int nK = n / 32, nN = (n + kN - 1) / kN;
      const int* sfn = slot_fn + sg;
      for (int j = 0; j < nN && ok; ++j) {
        const int nu0 = j * kN + (g >> 2), nu1 = j * kN + ((g + 128) >> 2);
        const int fnv0 = nu0 < n ? __ldg(sfn + nu0) : -1;
        const int fnv1 = (two && nu1 < n) ? __ldg(sfn + nu1) : -1;
        const int grp0 = g & 3, grp1 = (g + 128) & 3;
        for (int k = 0; k < nK; ++k, ++it) {
          const int sbb = it % kBStages;
          const int fmu_lane = __ldg(sfn + k * 32 + lane);
          if (it >= kBStages && !tc::mbar_wait(&S.b_empty[sbb], ((it / kBStages) - 1) & 1)) {
            ok = false;
            break;
          }
          unsigned long long w0[8], w1[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int f0 = __shfl_sync(0xffffffffu, fmu_lane, grp0 * 8 + u);
            const int f1 = __shfl_sync(0xffffffffu, fmu_lane, grp1 * 8 + u);
            w0[u] = (fnv0 >= 0 && f0 >= 0) ? __ldg(P8 + (int64_t)fnv0 * nbas + f0) : 0ull;
            w1[u] = (fnv1 >= 0 && f1 >= 0) ? __ldg(P8 + (int64_t)fnv1 * nbas + f1) : 0ull;
          }
#pragma unroll
          for (int sl = 0; sl < kSlices; ++sl) {
            *reinterpret_cast<unsigned long long*>(S.b[sbb] + sl * kBlkB + blk_off(g >> 2, grp0 * 8)) =
                gather_slice(w0, sl);
            if (two)
              *reinterpret_cast<unsigned long long*>(S.b[sbb] + sl * kBlkB + blk_off((g + 128) >> 2, grp1 * 8)) =
                  gather_slice(w1, sl);
          }
          tc::fence_proxy_async();
          tc::mbar_arrive(&S.b_full[sbb]);
        }
      }
    }
    if (!ok) atomicExch(err, 1);
  } else {  // epilogue: point row = 32 (warp & 3) + lane, columns 24 (warp >> 2) .. +24 of each slot block
    const int row = (warp & 3) * 32 + lane, half = warp >> 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16) + half * 24;
    int jj = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
      const int64_t sg = tso[t0 + ti];
      const int n = (int)(tso[t0 + ti + 1] - sg);
      const int nN = (n + kN - 1) / kN;
      const int* sfn = slot_fn + sg;
      const double rs = pow2(e_pt[ti * 128 + row] + kCombShift);
      double r_acc = 0.0, g_acc[3] = {0.0, 0.0, 0.0};
      for (int j = 0; j < nN && ok; ++j, ++jj) {
        const int b = jj & 1;
        if (!tc::mbar_wait(&S.acc_full[b], (jj >> 1) & 1)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        double x[24];
        read_acc24(trow + b * kAccCols, x);
        tc::fence_before_sync();
        tc::mbar_arrive(&S.acc_empty[b]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = (jj * 4 + u) * 2 + half, r = e % kERing;
          if (!tc::mbar_wait(&S.e_full[r], (e / kERing) & 1)) {
            ok = false;
            break;
          }
          const int c0 = j * kN + half * 24 + u * kECols;
          const double* eb = S.e[r];
#pragma unroll
          for (int v = 0; v < kECols; ++v) {
            const int c = c0 + v;
            if (c < n) {
              const int f = __ldg(sfn + c);
              const double X = f >= 0 ? x[u * kECols + v] * (rs * pow2(__ldg(e_P + f))) : 0.0;
              r_acc += X * eb[v * 128 + row];
              if (GGA) {
                g_acc[0] += X * eb[(kECols + v) * 128 + row];
                g_acc[1] += X * eb[(2 * kECols + v) * 128 + row];
                g_acc[2] += X * eb[(3 * kECols + v) * 128 + row];
              }
            }
          }
          tc::mbar_arrive(&S.e_empty[r]);
        }
      }
      if (!ok) break;
      const int64_t p = ti * 128 + row;
      atomicAdd(rho + p, r_acc);
      if (GGA) {
        atomicAdd(grx + p, 2.0 * g_acc[0]);
        atomicAdd(gry + p, 2.0 * g_acc[1]);
        atomicAdd(grz + p, 2.0 * g_acc[2]);
      }
    }
    if (!ok) atomicExch(err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

// ---------------------------------------------------------------------------
// Z and the V operand digits: warp per slot, lane = 4 consecutive points
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool GGA>
__global__ void __launch_bounds__(256, 2) k_sm_zquant(const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
                                                   const double* __restrict__ phi, const double* __restrict__ gx,
                                                   const double* __restrict__ gy, const double* __restrict__ gz,
                                                   const double* __restrict__ A, const double* __restrict__ Bx,
                                                   const double* __restrict__ By, const double* __restrict__ Bz,
                                                   int8_t* __restrict__ tZ, int8_t* __restrict__ tF,
                                                   int* __restrict__ e_Z, int* __restrict__ e_F) {
  __shared__ double sA[128], sB[3][128];
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < 128) {
    const int64_t p = (int64_t)blockIdx.x * 128 + tid;
    sA[tid] = A[p];
    if (GGA) {
      sB[0][tid] = Bx[p];
      sB[1][tid] = By[p];
      sB[2][tid] = Bz[p];
    }
  }
  __syncthreads();
  const int p0 = lane * 4;
  const int kstep = lane >> 3, kin = (lane & 7) * 4;
  const int64_t tile_off = sb * kDigBytesPerSlot;
  for (int i = warp; i < n; i += 8) {
    const int64_t o = (sb + i) * 128 + p0;
    double f[4], z[4];
    {
      const double2 a = *reinterpret_cast<const double2*>(phi + o);
      const double2 b = *reinterpret_cast<const double2*>(phi + o + 2);
      f[0] = a.x; f[1] = a.y; f[2] = b.x; f[3] = b.y;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) z[u] = sA[p0 + u] * f[u];
    if (GGA) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double* g = c == 0 ? gx : (c == 1 ? gy : gz);
        const double2 a = *reinterpret_cast<const double2*>(g + o);
        const double2 b = *reinterpret_cast<const double2*>(g + o + 2);
        z[0] += sB[c][p0] * a.x;
        z[1] += sB[c][p0 + 1] * a.y;
        z[2] += sB[c][p0 + 2] * b.x;
        z[3] += sB[c][p0 + 3] * b.y;
      }
    }
    const double mz = warp_max(fmax(fmax(fabs(z[0]), fabs(z[1])), fmax(fabs(z[2]), fabs(z[3]))));
    const double mf = warp_max(fmax(fmax(fabs(f[0]), fabs(f[1])), fmax(fabs(f[2]), fabs(f[3]))));
    const int ez = scale_exp(mz), ef = scale_exp(mf);
    if (lane == 0) {
      e_Z[sb + i] = ez;
      e_F[sb + i] = ef;
    }
    long long qz[4], qf[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      qz[u] = oz_int(z[u], ez);
      qf[u] = oz_int(f[u], ef);
    }
    uint32_t wz[kSlices], wf[kSlices];
    oz_pack4(qz, wz);
    oz_pack4(qf, wf);
#pragma unroll
    for (int sl = 0; sl < kSlices; ++sl) {
      const int64_t off = tile_off + (int64_t)(kstep * kSlices + sl) * n * 32 + blk_off(i, kin);
      *reinterpret_cast<uint32_t*>(tZ + off) = wz[sl];
      *reinterpret_cast<uint32_t*>(tF + off) = wf[sl];
    }
  }
}

// ---------------------------------------------------------------------------
// H[S_t, S_t] += Z_t^T phi_t, scatter-added into V (LDA: fn_i <= fn_j only,
// H is symmetric; GGA: the whole square, V = H + H^T when packing).
// Pairs of 128-slot row blocks I and 48-slot column blocks J, K = the tile's
// 128 points in 4 steps.  Persistent like k_sm_density.
// ---------------------------------------------------------------------------
struct VSmem {
  alignas(1024) int8_t a[kVStages][kOpA];
  alignas(1024) int8_t b[kVStages][kOpB];
  uint64_t full[kVStages];
  uint64_t empty[kVStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tslot;
};
constexpr int kVThreads = 320;  // warps 0-7 epilogue, 8 MMA, 9 producer

// first 48-slot block of pair row I: LDA needs columns j >= 128 I only
__device__ __forceinline__ int first_J(int I, bool all) { return all ? 0 : (kM * I) / kN; }

template <bool GGA>
__global__ void __launch_bounds__(kVThreads, 1)
    k_sm_vpot(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t nt, int64_t s0,
              const int8_t* __restrict__ tZ, const int8_t* __restrict__ tF, const int* __restrict__ e_Z,
              const int* __restrict__ e_F, double* __restrict__ V, int64_t ldv, int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  VSmem& S = *reinterpret_cast<VSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int s = 0; s < kVStages; ++s) {
      tc::mbar_init(&S.full[s], 1);
      tc::mbar_init(&S.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&S.acc_full[b], 1);
      tc::mbar_init(&S.acc_empty[b], 256);
    }
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  bool ok = true;
  if (warp == 9) {
    if (lane == 0) {  // producer: per pair and K step, Z rows of block I and phi rows of block J
      int it = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nI = (n + kM - 1) / kM, nJ = (n + kN - 1) / kN;
        const int8_t* zsrc = tZ + sb * kDigBytesPerSlot;
        const int8_t* fsrc = tF + sb * kDigBytesPerSlot;
        const int64_t blk = (int64_t)n * 32;  // bytes of one (K step, slice) block of the tile
        for (int I = 0; I < nI && ok; ++I)
          for (int J = first_J(I, GGA); J < nJ && ok; ++J)
            for (int k = 0; k < 4; ++k, ++it) {
              const int s = it % kVStages;
              if (it >= kVStages && !tc::mbar_wait(&S.empty[s], ((it / kVStages) - 1) & 1)) {
                ok = false;
                break;
              }
              tc::mbar_expect_tx(&S.full[s], kOpA + kOpB);
              for (int sl = 0; sl < kSlices; ++sl) {
                tc::bulk_g2s(S.a[s] + sl * kBlkA, zsrc + (k * kSlices + sl) * blk + (int64_t)I * kM * 32, kBlkA,
                             &S.full[s]);
                tc::bulk_g2s(S.b[s] + sl * kBlkB, fsrc + (k * kSlices + sl) * blk + (int64_t)J * kN * 32, kBlkB,
                             &S.full[s]);
              }
            }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 8) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = tc::idesc_s8(kM, kN);
      int it = 0, pp = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nI = (n + kM - 1) / kM, nJ = (n + kN - 1) / kN;
        for (int I = 0; I < nI && ok; ++I)
          for (int J = first_J(I, GGA); J < nJ && ok; ++J, ++pp) {
            const int b = pp & 1;
            if (pp >= 2 && !tc::mbar_wait(&S.acc_empty[b], ((pp >> 1) - 1) & 1)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
            for (int k = 0; k < 4; ++k, ++it) {
              const int s = it % kVStages;
              if (!tc::mbar_wait(&S.full[s], (it / kVStages) & 1)) {
                ok = false;
                break;
              }
              tc::fence_after_sync();
              oz_mma_pairs(tbase + b * kAccCols, kN, tc::smem_u32(S.a[s]), kBlkA, tc::smem_u32(S.b[s]), kBlkB,
                           idesc, k == 0);
              tc::mma_commit(&S.empty[s]);
            }
            tc::mma_commit(&S.acc_full[b]);
          }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else {  // epilogue: slot row i = 128 I + 32 (warp & 3) + lane, columns 24 (warp >> 2) .. of each block
    const int half = warp >> 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16) + half * 24;
    int pp = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
      const int64_t sg = tso[t0 + ti];
      const int64_t sb = sg - s0;
      const int n = (int)(tso[t0 + ti + 1] - sg);
      const int nI = (n + kM - 1) / kM, nJ = (n + kN - 1) / kN;
      const int* sfn = slot_fn + sg;
      for (int I = 0; I < nI && ok; ++I) {
        const int i = I * kM + (warp & 3) * 32 + lane;
        const int fi = i < n ? __ldg(sfn + i) : -1;
        const int ezi = i < n ? __ldg(e_Z + sb + i) : 0;
        for (int J = first_J(I, GGA); J < nJ; ++J, ++pp) {
          const int b = pp & 1;
          if (!tc::mbar_wait(&S.acc_full[b], (pp >> 1) & 1)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          double x[24];
          read_acc24(trow + b * kAccCols, x);
          tc::fence_before_sync();
          tc::mbar_arrive(&S.acc_empty[b]);
          if (fi < 0) continue;
          const int j0 = J * kN + half * 24;
#pragma unroll
          for (int c = 0; c < 24; ++c) {
            const int j = j0 + c;
            const int fj = j < n ? __ldg(sfn + j) : -1;
            if (fj >= 0 && (GGA || fj >= fi))
              atomicAdd(V + (int64_t)fi * ldv + fj, x[c] * pow2(ezi + __ldg(e_F + sb + j) + kCombShift));
          }
        }
      }
    }
    if (!ok) atomicExch(err, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

}  // namespace

int64_t screen_mixed_bytes_per_slot() { return 3 * kDigBytesPerSlot + 8; }
int64_t screen_mixed_bytes_per_tile() { return 128 * 4; }

int screen_mixed_create(ScreenMixed** out, const ScreenMixedInput& in, std::string& err) {
  *out = nullptr;
  ScreenMixed* m = new ScreenMixed();
  m->nbas = in.nbas;
  m->ldc = in.ldc;
  m->gga = in.gga;
  m->chunk_slots = in.chunk_slots;
  m->chunk_tiles = in.chunk_tiles;
  m->max_n = in.max_n;
  cudaError_t e = cudaSuccess;
  const size_t dig = (size_t)in.chunk_slots * kDigBytesPerSlot;
  if (e == cudaSuccess) e = sm_alloc(m, &m->P8, (size_t)in.nbas * in.nbas);
  if (e == cudaSuccess) e = sm_alloc(m, &m->e_P, (size_t)in.nbas);
  if (e == cudaSuccess) e = sm_alloc(m, &m->tA, dig);
  if (e == cudaSuccess) e = sm_alloc(m, &m->tZ, dig);
  if (e == cudaSuccess) e = sm_alloc(m, &m->tF, dig);
  if (e == cudaSuccess) e = sm_alloc(m, &m->e_pt, (size_t)in.chunk_tiles * 128);
  if (e == cudaSuccess) e = sm_alloc(m, &m->e_Z, (size_t)in.chunk_slots);
  if (e == cudaSuccess) e = sm_alloc(m, &m->e_F, (size_t)in.chunk_slots);
  if (e == cudaSuccess) e = sm_alloc(m, &m->err, 1);
  // the slack rows after a chunk's last slot are read (never used) by whole-block copies
  if (e == cudaSuccess) e = cudaMemset(m->tA, 0, dig);
  if (e == cudaSuccess) e = cudaMemset(m->tZ, 0, dig);
  if (e == cudaSuccess) e = cudaMemset(m->tF, 0, dig);
  if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
  if (e != cudaSuccess) {
    err = std::string("screened mixed-precision buffers: ") + cudaGetErrorString(e);
    screen_mixed_destroy(m);
    return e == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA;
  }
  const int dsm = (int)sizeof(DensSmem), vsm = (int)sizeof(VSmem);
  cudaFuncSetAttribute(k_sm_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_density<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_vpot<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, vsm);
  e = cudaFuncSetAttribute(k_sm_vpot<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, vsm);
  int dev = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    err = std::string("screened mixed-precision kernels: ") + cudaGetErrorString(e) +
          " (a tile lists too many functions for shared memory)";
    screen_mixed_destroy(m);
    return PGXC_ENOTSUP;
  }
  *out = m;
  return PGXC_OK;
}

void screen_mixed_destroy(ScreenMixed* m) {
  if (!m) return;
  for (void* p : m->allocs) cudaFree(p);
  delete m;
}

int screen_mixed_prepare(ScreenMixed* m, const BuildArgs& a, cudaStream_t st) {
  k_sm_rowexp_P<<<(unsigned)m->nbas, 256, 0, st>>>(a.P, a.ldc, m->nbas, m->e_P);
  const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((m->nbas * m->nbas + 255) / 256, 148 * 16));
  k_sm_quant_P<<<nb, 256, 0, st>>>(a.P, a.ldc, m->nbas, m->e_P, m->P8);
  return 2;
}

int screen_mixed_basis(ScreenMixed* m, const int64_t* tso, int64_t t0, int64_t nt, int64_t s0, const double* phi,
                       cudaStream_t st) {
  k_sm_quant_pts<<<(unsigned)nt, 128, 0, st>>>(tso, t0, s0, phi, m->e_pt, m->tA);
  return 1;
}

int screen_mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                         const double* phi, const double* gx, const double* gy, const double* gz, double* rho,
                         double* grx, double* gry, double* grz, cudaStream_t st) {
  cudaMemsetAsync(rho, 0, sizeof(double) * nt * 128, st);
  if (m->gga) {
    cudaMemsetAsync(grx, 0, sizeof(double) * nt * 128, st);
    cudaMemsetAsync(gry, 0, sizeof(double) * nt * 128, st);
    cudaMemsetAsync(grz, 0, sizeof(double) * nt * 128, st);
  }
  const unsigned grid = (unsigned)std::min<int64_t>(nt, m->nsm);
  const int smem = (int)sizeof(DensSmem);
  if (m->gga)
    k_sm_density<true><<<grid, kDensThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, m->tA, m->e_pt, m->P8, m->e_P,
                                                         m->nbas, phi, gx, gy, gz, rho, grx, gry, grz, m->err);
  else
    k_sm_density<false><<<grid, kDensThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, m->tA, m->e_pt, m->P8, m->e_P,
                                                          m->nbas, phi, nullptr, nullptr, nullptr, rho, nullptr,
                                                          nullptr, nullptr, m->err);
  return 1;
}

int screen_mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, const int* slot_tile, int64_t t0,
                           int64_t nt, int64_t s0, int64_t ns, const double* phi, const double* gx, const double* gy,
                           const double* gz, const double* A, const double* Bx, const double* By, const double* Bz,
                           double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1) {
  (void)slot_tile;
  (void)ns;
  if (m->gga)
    k_sm_zquant<true><<<(unsigned)nt, 256, 0, st>>>(tso, t0, s0, phi, gx, gy, gz, A, Bx, By, Bz, m->tZ, m->tF,
                                                    m->e_Z, m->e_F);
  else
    k_sm_zquant<false><<<(unsigned)nt, 256, 0, st>>>(tso, t0, s0, phi, nullptr, nullptr, nullptr, A, nullptr,
                                                     nullptr, nullptr, m->tZ, m->tF, m->e_Z, m->e_F);
  cudaEventRecord(k0, st);
  const unsigned grid = (unsigned)std::min<int64_t>(nt, m->nsm);
  const int smem = (int)sizeof(VSmem);
  if (m->gga)
    k_sm_vpot<true><<<grid, kVThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, m->tZ, m->tF, m->e_Z, m->e_F, V, ldv,
                                                   m->err);
  else
    k_sm_vpot<false><<<grid, kVThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, m->tZ, m->tF, m->e_Z, m->e_F, V, ldv,
                                                    m->err);
  cudaEventRecord(k1, st);
  return 2;
}

int screen_mixed_error_flag(ScreenMixed* m, cudaStream_t st, int* flag) {
  int h = 0;
  if (cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return PGXC_ECUDA;
  if (cudaMemsetAsync(m->err, 0, sizeof(int), st) != cudaSuccess) return PGXC_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return PGXC_ECUDA;
  *flag = h;
  return PGXC_OK;
}

}  // namespace pgxc
