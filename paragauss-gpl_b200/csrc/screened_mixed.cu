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
constexpr int kDStages = 4;
constexpr int kVStages = 4;
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
      int8_t d[kSlices][16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        int8_t q[kSlices];
        digits(src[(int64_t)(kb * 32 + h * 16 + k) * 128], e, q);
#pragma unroll
        for (int s = 0; s < kSlices; ++s) d[s][k] = q[s];
      }
#pragma unroll
      for (int s = 0; s < kSlices; ++s)
        *reinterpret_cast<uint4*>(dst + (int64_t)kb * kOpA + s * kBlkA + blk_off(p, h * 16)) =
            *reinterpret_cast<const uint4*>(d[s]);
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
struct DensSmem {
  alignas(1024) int8_t a[kDStages][kOpA];
  alignas(1024) int8_t b[kDStages][kOpB];
  double red[4][128];
  uint64_t full[kDStages];
  uint64_t empty[kDStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tslot;
};
constexpr int kDensThreads = 448;  // warps 0-7 epilogue, 8 MMA, 9 A copies, 10-13 B gather

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

template <bool GGA>
__global__ void __launch_bounds__(kDensThreads, 1)
    k_sm_density(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t s0,
                 const int8_t* __restrict__ tA, const int* __restrict__ e_pt,
                 const unsigned long long* __restrict__ P8, const int* __restrict__ e_P, int64_t nbas,
                 const double* __restrict__ phi, const double* __restrict__ gx, const double* __restrict__ gy,
                 const double* __restrict__ gz, double* __restrict__ rho, double* __restrict__ grx,
                 double* __restrict__ gry, double* __restrict__ grz, int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  DensSmem& S = *reinterpret_cast<DensSmem*>(smem_raw);
  int* sfn = reinterpret_cast<int*>(smem_raw + sizeof(DensSmem));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int nK = n / 32, nN = (n + kN - 1) / kN, total = nK * nN;
  for (int i = tid; i < n; i += blockDim.x) sfn[i] = slot_fn[tso[t] + i];
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int s = 0; s < kDStages; ++s) {
      tc::mbar_init(&S.full[s], 1 + 128);
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
  double r_acc = 0.0, g_acc[3] = {0.0, 0.0, 0.0};
  if (warp == 8) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = tc::idesc_s8(kM, kN);
      int it = 0;
      for (int j = 0; j < nN && ok; ++j) {
        const int b = j & 1;
        if (j >= 2 && !tc::mbar_wait(&S.acc_empty[b], ((j >> 1) - 1) & 1)) ok = false;
        tc::fence_after_sync();
        for (int k = 0; k < nK && ok; ++k, ++it) {
          const int s = it % kDStages;
          if (!tc::mbar_wait(&S.full[s], (it / kDStages) & 1)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          oz_mma_pairs(tbase + b * kAccCols, kN, tc::smem_u32(S.a[s]), kBlkA, tc::smem_u32(S.b[s]), kBlkB, idesc,
                       k == 0);
          tc::mma_commit(&S.empty[s]);
        }
        tc::mma_commit(&S.acc_full[b]);  // also after a failed wait: releases the epilogue
      }
      if (!ok) {
        atomicExch(err, 1);
        for (int j = 0; j < nN; ++j) tc::mma_commit(&S.acc_full[j & 1]);
      }
    }
  } else if (warp == 9) {
    if (lane == 0) {  // A producer: the tile's digits of phi, one 32-slot K block per stage
      const int8_t* src = tA + sb * kDigBytesPerSlot;
      for (int it = 0; it < total && ok; ++it) {
        const int s = it % kDStages, k = it % nK;
        if (it >= kDStages && !tc::mbar_wait(&S.empty[s], ((it / kDStages) - 1) & 1)) ok = false;
        if (!ok) break;
        tc::mbar_expect_tx(&S.full[s], kOpA);
        tc::bulk_g2s(S.a[s], src + (int64_t)k * kOpA, kOpA, &S.full[s]);
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp >= 10) {  // B producers: P8[fn(nu)][fn(mu)] gathered into the K-major digit block
    const int g = tid - 320;
    for (int it = 0; it < total && ok; ++it) {
      const int s = it % kDStages, j = it / nK, k = it % nK;
      if (it >= kDStages && !tc::mbar_wait(&S.empty[s], ((it / kDStages) - 1) & 1)) {
        ok = false;
        break;
      }
      for (int task = g; task < kN * 4; task += 128) {
        const int r = task >> 2, grp = task & 3;
        const int nu = j * kN + r;
        const int fnv = nu < n ? sfn[nu] : -1;
        unsigned long long w[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int fmu = sfn[k * 32 + grp * 8 + u];
          w[u] = (fnv >= 0 && fmu >= 0) ? __ldg(P8 + (int64_t)fnv * nbas + fmu) : 0ull;
        }
#pragma unroll
        for (int sl = 0; sl < kSlices; ++sl)
          *reinterpret_cast<unsigned long long*>(S.b[s] + sl * kBlkB + blk_off(r, grp * 8)) = gather_slice(w, sl);
      }
      tc::fence_proxy_async();
      tc::mbar_arrive(&S.full[s]);
    }
    if (!ok) atomicExch(err, 1);
  } else {  // epilogue: point row = 32 (warp & 3) + lane, columns 24 (warp >> 2) .. +24 of each slot block
    const int row = (warp & 3) * 32 + lane, half = warp >> 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16) + half * 24;
    const double rs = pow2(e_pt[(int64_t)blockIdx.x * 128 + row] + kCombShift);
    for (int j = 0; j < nN; ++j) {
      const int b = j & 1;
      if (!tc::mbar_wait(&S.acc_full[b], (j >> 1) & 1)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      double x[24];
      read_acc24(trow + b * kAccCols, x);
      tc::fence_before_sync();
      tc::mbar_arrive(&S.acc_empty[b]);
      const int c0 = j * kN + half * 24;
#pragma unroll
      for (int cc = 0; cc < 24; cc += 4) {
        if (c0 + cc >= n) break;
        double v[4], w0[4], w1[4], w2[4], sc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int c = c0 + cc + u;  // n is a multiple of 32, so c < n for the whole group of 4
          const int64_t o = (sb + c) * 128 + row;
          const int f = sfn[c];
          sc[u] = f >= 0 ? pow2(__ldg(e_P + f)) : 0.0;
          v[u] = __ldg(phi + o);
          if (GGA) {
            w0[u] = __ldg(gx + o);
            w1[u] = __ldg(gy + o);
            w2[u] = __ldg(gz + o);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double X = x[cc + u] * (rs * sc[u]);
          r_acc += X * v[u];
          if (GGA) {
            g_acc[0] += X * w0[u];
            g_acc[1] += X * w1[u];
            g_acc[2] += X * w2[u];
          }
        }
      }
    }
    if (!ok) atomicExch(err, 1);
  }
  // combine the two column halves of each point
  if (warp >= 4 && warp < 8) {
    const int row = (warp & 3) * 32 + lane;
    S.red[0][row] = r_acc;
    S.red[1][row] = g_acc[0];
    S.red[2][row] = g_acc[1];
    S.red[3][row] = g_acc[2];
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp < 4) {
    const int row = warp * 32 + lane;
    const int64_t p = (int64_t)blockIdx.x * 128 + row;
    rho[p] = r_acc + S.red[0][row];
    if (GGA) {
      grx[p] = 2.0 * (g_acc[0] + S.red[1][row]);
      gry[p] = 2.0 * (g_acc[1] + S.red[2][row]);
      grz[p] = 2.0 * (g_acc[2] + S.red[3][row]);
    }
  }
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
__global__ void __launch_bounds__(256) k_sm_zquant(const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
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
      const double* gs[3] = {gx, gy, gz};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 a = *reinterpret_cast<const double2*>(gs[c] + o);
        const double2 b = *reinterpret_cast<const double2*>(gs[c] + o + 2);
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
    int8_t dz[4][kSlices], df[4][kSlices];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      digits(z[u], ez, dz[u]);
      digits(f[u], ef, df[u]);
    }
#pragma unroll
    for (int sl = 0; sl < kSlices; ++sl) {
      const int64_t off = tile_off + (int64_t)(kstep * kSlices + sl) * n * 32 + blk_off(i, kin);
      uint32_t wz = 0, wf = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        wz |= (uint32_t)(uint8_t)dz[u][sl] << (8 * u);
        wf |= (uint32_t)(uint8_t)df[u][sl] << (8 * u);
      }
      *reinterpret_cast<uint32_t*>(tZ + off) = wz;
      *reinterpret_cast<uint32_t*>(tF + off) = wf;
    }
  }
}

// ---------------------------------------------------------------------------
// H[S_t, S_t] += Z_t^T phi_t, scatter-added into V
// ---------------------------------------------------------------------------
struct VSmem {
  alignas(1024) int8_t a[4][kOpA];          // the Z digits of one 128-slot block, all 4 K steps
  int8_t pad_[8192];                        // keeps one CTA per SM (each holds all 512 TMEM columns)
  alignas(1024) int8_t b[kVStages][kOpB];   // phi digits of one 48-slot block, one K step
  uint64_t a_full, a_empty;
  uint64_t b_full[kVStages];
  uint64_t b_empty[kVStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tslot;
};
constexpr int kVThreads = 320;  // warps 0-7 epilogue, 8 MMA, 9 producer

// first 48-slot block with a column j >= 128 I (LDA keeps j >= i only)
__device__ __forceinline__ int first_J(int I, bool all) { return all ? 0 : (kM * I) / kN; }

template <bool GGA>
__global__ void __launch_bounds__(kVThreads, 1)
    k_sm_vpot(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t s0,
              const int8_t* __restrict__ tZ, const int8_t* __restrict__ tF, const int* __restrict__ e_Z,
              const int* __restrict__ e_F, double* __restrict__ V, int64_t ldv, int* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  VSmem& S = *reinterpret_cast<VSmem*>(smem_raw);
  int* sfn = reinterpret_cast<int*>(smem_raw + sizeof(VSmem));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int nI = (n + kM - 1) / kM, nJ = (n + kN - 1) / kN;
  for (int i = tid; i < n; i += blockDim.x) sfn[i] = slot_fn[tso[t] + i];
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    tc::mbar_init(&S.a_full, 1);
    tc::mbar_init(&S.a_empty, 1);
    for (int s = 0; s < kVStages; ++s) {
      tc::mbar_init(&S.b_full[s], 1);
      tc::mbar_init(&S.b_empty[s], 1);
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
  const int8_t* zsrc = tZ + sb * kDigBytesPerSlot;
  const int8_t* fsrc = tF + sb * kDigBytesPerSlot;
  const int64_t blk = (int64_t)n * 32;  // bytes of one (K step, slice) block of the tile
  bool ok = true;
  if (warp == 9) {
    if (lane == 0) {  // producer
      int pi = 0;
      for (int I = 0; I < nI && ok; ++I) {
        if (I > 0 && !tc::mbar_wait(&S.a_empty, (I - 1) & 1)) {
          ok = false;
          break;
        }
        tc::mbar_expect_tx(&S.a_full, 4 * kOpA);
        for (int k = 0; k < 4; ++k)
          for (int sl = 0; sl < kSlices; ++sl)
            tc::bulk_g2s(S.a[k] + sl * kBlkA, zsrc + (k * kSlices + sl) * blk + (int64_t)I * kM * 32, kBlkA,
                         &S.a_full);
        for (int J = first_J(I, GGA); J < nJ && ok; ++J, ++pi) {
          for (int k = 0; k < 4; ++k) {
            const int ib = pi * 4 + k, s = ib % kVStages;
            if (ib >= kVStages && !tc::mbar_wait(&S.b_empty[s], ((ib / kVStages) - 1) & 1)) {
              ok = false;
              break;
            }
            tc::mbar_expect_tx(&S.b_full[s], kOpB);
            for (int sl = 0; sl < kSlices; ++sl)
              tc::bulk_g2s(S.b[s] + sl * kBlkB, fsrc + (k * kSlices + sl) * blk + (int64_t)J * kN * 32, kBlkB,
                           &S.b_full[s]);
          }
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 8) {
    if (lane == 0) {  // MMA issuer
      const uint32_t idesc = tc::idesc_s8(kM, kN);
      int pi = 0;
      for (int I = 0; I < nI && ok; ++I) {
        if (!tc::mbar_wait(&S.a_full, I & 1)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        for (int J = first_J(I, GGA); J < nJ && ok; ++J, ++pi) {
          const int b = pi & 1;
          if (pi >= 2 && !tc::mbar_wait(&S.acc_empty[b], ((pi >> 1) - 1) & 1)) ok = false;
          tc::fence_after_sync();
          for (int k = 0; k < 4 && ok; ++k) {
            const int ib = pi * 4 + k, s = ib % kVStages;
            if (!tc::mbar_wait(&S.b_full[s], (ib / kVStages) & 1)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
            oz_mma_pairs(tbase + b * kAccCols, kN, tc::smem_u32(S.a[k]), kBlkA, tc::smem_u32(S.b[s]), kBlkB, idesc,
                         k == 0);
            tc::mma_commit(&S.b_empty[s]);
          }
          tc::mma_commit(&S.acc_full[b]);
        }
        tc::mma_commit(&S.a_empty);
      }
      if (!ok) {
        atomicExch(err, 1);
        for (int q = 0; q < 2; ++q) tc::mma_commit(&S.acc_full[q]);
      }
    }
  } else {  // epilogue: slot row i = 128 I + 32 (warp & 3) + lane, columns 24 (warp >> 2) .. of each block
    const int half = warp >> 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16) + half * 24;
    int pi = 0;
    for (int I = 0; I < nI && ok; ++I) {
      const int i = I * kM + (warp & 3) * 32 + lane;
      const int fi = i < n ? sfn[i] : -1;
      const int ez = i < n ? e_Z[sb + i] : 0;
      for (int J = first_J(I, GGA); J < nJ; ++J, ++pi) {
        const int b = pi & 1;
        if (!tc::mbar_wait(&S.acc_full[b], (pi >> 1) & 1)) {
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
          const int fj = j < n ? sfn[j] : -1;
          if (fj >= 0 && (GGA || fj >= fi))
            atomicAdd(V + (int64_t)fi * ldv + fj, x[c] * pow2(ez + __ldg(e_F + sb + j) + kCombShift));
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
  const int dsm = (int)sizeof(DensSmem) + 4 * in.max_n;
  const int vsm = (int)sizeof(VSmem) + 4 * in.max_n;
  cudaFuncSetAttribute(k_sm_density<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_density<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_vpot<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, vsm);
  e = cudaFuncSetAttribute(k_sm_vpot<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, vsm);
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
  const int smem = (int)sizeof(DensSmem) + 4 * m->max_n;
  if (m->gga)
    k_sm_density<true><<<(unsigned)nt, kDensThreads, smem, st>>>(tso, slot_fn, t0, s0, m->tA, m->e_pt, m->P8,
                                                                 m->e_P, m->nbas, phi, gx, gy, gz, rho, grx, gry,
                                                                 grz, m->err);
  else
    k_sm_density<false><<<(unsigned)nt, kDensThreads, smem, st>>>(tso, slot_fn, t0, s0, m->tA, m->e_pt, m->P8,
                                                                  m->e_P, m->nbas, phi, nullptr, nullptr, nullptr,
                                                                  rho, nullptr, nullptr, nullptr, m->err);
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
  const int smem = (int)sizeof(VSmem) + 4 * m->max_n;
  if (m->gga)
    k_sm_vpot<true><<<(unsigned)nt, kVThreads, smem, st>>>(tso, slot_fn, t0, s0, m->tZ, m->tF, m->e_Z, m->e_F, V,
                                                           ldv, m->err);
  else
    k_sm_vpot<false><<<(unsigned)nt, kVThreads, smem, st>>>(tso, slot_fn, t0, s0, m->tZ, m->tF, m->e_Z, m->e_F, V,
                                                            ldv, m->err);
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
