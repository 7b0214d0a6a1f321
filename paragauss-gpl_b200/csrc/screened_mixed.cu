// screened_mixed.cu -- INT8 tensor-core stages of the screened XC build.
//
// Both contractions of a tile run on tcgen05.mma kind::i8 with the Ozaki
// split of ozaki.cuh (15 digit-pair products per K step issued as 5 MMAs of
// N = 240..48, exact INT32 accumulation in TMEM, FP64 combination):
//
//   k_sm_quant_pts   phi_t -> INT8 digits, one scale per point          (A of X)
//   k_sm_rowexp_P,   P -> packed digits P8[nu][mu] (5 bytes of a 64-bit
//   k_sm_quant_P     word), one scale per row nu                       (B of X)
//   k_sm_density     X = phi_t P[S_t, S_t], 128 points x 48 slots per MMA;
//                    A by bulk copy, B gathered from P8 by four producer
//                    warps, two TMEM accumulator sets (MMA of slot block j+1
//                    overlaps the epilogue of block j); fused FP64 epilogue
//                    rho += X phi, grad rho += 2 X grad phi
//   k_sm_zquant      Z = A phi (+ B . grad phi) in FP64 and the digits of phi
//                    (slice-interleaved per 8 slots: one copy per A block) and
//                    of Z (slices one after another), one scale per
//                    (tile, slot)                                       (A, B of V)
//   k_sm_vpot        H[S_t, S_t] += Z_t^T phi_t computed as phi_t Z_t^T (TMEM
//                    lane = column j of H), 128 x 48 slot blocks, K = the
//                    tile's 128 points; scaled in FP64 and scatter-added
//                    into the full matrix with atomics that run along rows
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
constexpr int kDStages = 4;                // density: operand ring (A and gathered B of one K step)
constexpr int kDigBytesPerSlot = 640;      // 128 points x 5 slices

}  // namespace

struct ScreenMixed {
  int64_t nbas = 0, ldc = 0;
  bool gga = false;
  int64_t chunk_slots = 0, chunk_tiles = 0;
  int max_n = 0;
  int nspin = 1;
  unsigned long long* P8[2] = {};    // [nbas][nbas] per spin
  int* e_P[2] = {};                  // [nbas] per spin
  int8_t* tA = nullptr;              // density A digits, [slot block of 32][slice][128 x 32] per tile
  int8_t* tB = nullptr;              // density B digits, [stage][slice][48 x 32] per tile
  const int64_t* b_off = nullptr;    // [ntiles + 1] first B stage of each tile
  int* e_pt = nullptr;               // [chunk_tiles * 128]
  int8_t* tF = nullptr;              // V operand A (phi), [kstep][8-slot group][slice][8 x 32] per tile
  int8_t* tZ = nullptr;              // V operand B (Z), [kstep][slice][n x 32] per tile
  double* zs = nullptr;              // [chunk_slots] 2^e of each slot's Z digits
  double* fs = nullptr;              // [chunk_slots] 2^(e - 40) of each slot's phi digits (the combine shift folded in)
  double* ps = nullptr;              // [chunk_slots] 2^e_P of each slot's function (0 for padding)
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
// |phi| over the tile's slots, from pmax)
__global__ void __launch_bounds__(128) k_sm_quant_pts(const int64_t* __restrict__ tso, int64_t t0, int64_t s0,
                                                      const double* __restrict__ phi,
                                                      const unsigned long long* __restrict__ pmax,
                                                      int* __restrict__ e_pt, int8_t* __restrict__ tA) {
  const int64_t t = t0 + blockIdx.x;
  const int64_t sb = tso[t] - s0;
  const int n = (int)(tso[t + 1] - tso[t]);
  const int p = threadIdx.x;
  const double* src = phi + sb * 128 + p;
  // largest |phi| of the point over the tile's slots, recorded by the basis kernel
  const int e = scale_exp(__longlong_as_double((long long)pmax[(int64_t)blockIdx.x * 128 + p]));
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
// B operand of the density contraction, per tile: for slot block j (48 rows
// nu) and K step k (32 slots mu) the 5 digit slices of P[fn(nu)][fn(mu)] in
// the K-major MMA layout, stored at stage b_off[t] + j nK + k; rows past the
// tile's slots are zero.  One block per tile, thread = (row, 8 K values).
// ---------------------------------------------------------------------------
constexpr int kGatherSplit = 4;  // blocks per tile: block y takes the slot blocks j = y, y + 4, ...
__global__ void __launch_bounds__(kBlock4(192)) k_sm_gather_B(const int64_t* __restrict__ tso,
                                                    const int* __restrict__ slot_fn,
                                                    const int64_t* __restrict__ b_off, int64_t t0, int64_t s0,
                                                    const unsigned long long* __restrict__ P8,
                                                    const int* __restrict__ e_P, int64_t nbas,
                                                    int8_t* __restrict__ tB, double* __restrict__ ps,
                                                    const int* __restrict__ tile_mol,
                                                    const SetMolDev* __restrict__ mols) {
  extern __shared__ int sfn[];
  const int64_t t = t0 + blockIdx.x;
  if (tile_mol) {  // a set: this tile's context
    const SetMolDev& M = mols[tile_mol[t]];
    P8 = M.P8;
    e_P = M.e_P;
    nbas = M.nbas;
  }
  const int64_t sg = tso[t];
  const int n = (int)(tso[t + 1] - sg);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int f = slot_fn[sg + i];
    sfn[i] = f;
    if (blockIdx.y == 0) ps[sg - s0 + i] = f >= 0 ? pow2(e_P[f]) : 0.0;  // P's row scale for the density epilogue
  }
  __syncthreads();
  if (threadIdx.x >= 192) return;  // thread = (row of 48, group of 8 K values)
  const int nK = n / 32, nN = (n + kN - 1) / kN;
  const int r = threadIdx.x >> 2, grp = threadIdx.x & 3;
  int8_t* out = tB + (b_off[t] - b_off[t0]) * kOpB;
  for (int j = blockIdx.y; j < nN; j += kGatherSplit) {
    const int nu = j * kN + r;
    const int fnv = nu < n ? sfn[nu] : -1;
    const unsigned long long* prow = P8 + (int64_t)max(fnv, 0) * nbas;
    for (int k = 0; k < nK; k += 2) {  // two K steps per pass: 16 loads in flight (nK is even or ends the loop)
      unsigned long long w[2][8];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int kk = min(k + h, nK - 1);
          const int fmu = sfn[kk * 32 + grp * 8 + u];
          w[h][u] = (fnv >= 0 && fmu >= 0) ? __ldg(prow + fmu) : 0ull;
        }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (k + h >= nK) break;
        int8_t* o = out + (int64_t)(j * nK + k + h) * kOpB;
#pragma unroll
        for (int sl = 0; sl < kSlices; ++sl)
          *reinterpret_cast<unsigned long long*>(o + sl * kBlkB + blk_off(r, grp * 8)) = gather_slice(w[h], sl);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// X = phi_t P[S_t, S_t] with fused rho / grad rho
// ---------------------------------------------------------------------------
// epilogue operands: phi (and grad phi) of 4 slots x 128 points per buffer;
// the 12 epilogue warps take the three 16-column thirds of each 48-slot
// block, and each third has two ring buffers
constexpr int kECols = 4;
constexpr int kEThirds = 3;
constexpr int kERing = 2 * kEThirds;
constexpr int kEGroups = kN / kEThirds / kECols;  // staged groups per column third of a slot block
constexpr int kEBuf = 4 * kECols * 128;           // doubles
struct DensSmem {
  alignas(1024) int8_t a[kDStages][kOpA];
  alignas(1024) int8_t b[kDStages][kOpB];
  alignas(128) double e[kERing][kEBuf];   // [array][column][point]
  uint64_t full[kDStages];
  uint64_t empty[kDStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t e_full[kERing];
  uint64_t e_empty[kERing];
  uint32_t tslot;
};
// warps 0-7 and 11-14 epilogue (three per TMEM lane quarter), 8 MMA, 9 operand
// copies, 10 epilogue-operand copies, 15 idle
constexpr int kDensThreads = tc::kWholeSmThreads;
constexpr int kDensEpiWarps = 12;

// TMEM -> the W combined FP64 values of W consecutive columns of one
// accumulator set (taddr: the first of them in group 0, at this warp's lane
// quarter; the five digit groups are kN columns apart).
template <int W>
__device__ __forceinline__ void acc_cols(uint32_t taddr, double* x) {
  uint32_t r[kGroups][W];
#pragma unroll
  for (int g = 0; g < kGroups; ++g) {
    if constexpr (W == 16) tc::tmem_ld16u(taddr + g * kN, r[g]);
    else if constexpr (W == 8) tc::tmem_ld8(taddr + g * kN, r[g]);
    else tc::tmem_ld4(taddr + g * kN, r[g]);
  }
  tc::tmem_ld_wait();
#pragma unroll
  for (int g = 0; g < kGroups; ++g) tc::tmem_regs_ready(r[g]);
#pragma unroll
  for (int c = 0; c < W; ++c) {
    uint32_t v[kGroups];
#pragma unroll
    for (int g = 0; g < kGroups; ++g) v[g] = r[g][c];
    x[c] = oz_combine(v);
  }
}
// Persistent: CTA c takes the chunk's tiles c, c + G, c + 2G, ... (G = grid
// size); the copy / MMA / epilogue pipeline runs on across tile boundaries.
// rho and grad rho are accumulated with atomics (the two column halves of a
// point and nothing else), so they must be zero on entry.
// GT: element type of the grad phi planes (staged beside phi in the same
// ring entry: phi in doubles, then the three gradient blocks in GT).
template <bool GGA, typename GT>
__global__ void __launch_bounds__(kDensThreads, 1)
    k_sm_density(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t nt,
                 int64_t s0, const int8_t* __restrict__ tA, const int* __restrict__ e_pt,
                 const int8_t* __restrict__ tB, const int64_t* __restrict__ b_off, const double* __restrict__ ps,
                 const double* __restrict__ phi, const GT* __restrict__ gx, const GT* __restrict__ gy,
                 const GT* __restrict__ gz, double* __restrict__ rho, double* __restrict__ grx,
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
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&S.acc_full[b], 1);
      tc::mbar_init(&S.acc_empty[b], 32 * kDensEpiWarps);
    }
    for (int r = 0; r < kERing; ++r) {
      tc::mbar_init(&S.e_full[r], 1);
      tc::mbar_init(&S.e_empty[r], 128);  // the four warps of one column third
    }
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  bool ok = true;
  if (warp == 10) {
    if (lane == 0) {  // epilogue operands: per slot block j, group u, third h: kECols slots of phi (grad phi)
      int e = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nN = (n + kN - 1) / kN;
        for (int j = 0; j < nN && ok; ++j) {
          for (int u = 0; u < kEGroups && ok; ++u)
            for (int h = 0; h < kEThirds; ++h, ++e) {
              const int r = e % kERing;
              if (e >= kERing && !tc::mbar_wait(&S.e_empty[r], ((e / kERing) - 1) & 1)) {
                ok = false;
                break;
              }
              const int c0 = j * kN + h * (kN / kEThirds) + u * kECols;
              const int nc = max(0, min(kECols, n - c0));
              if (nc == 0) {
                tc::mbar_arrive(&S.e_full[r]);
                continue;
              }
              const uint32_t bytes = (uint32_t)nc * 128 * sizeof(double);
              const uint32_t gbytes = (uint32_t)nc * 128 * sizeof(GT);
              const int64_t off = (sb + c0) * 128;
              tc::mbar_expect_tx(&S.e_full[r], bytes + (GGA ? 3 * gbytes : 0));
              tc::bulk_g2s(S.e[r], phi + off, bytes, &S.e_full[r]);
              if (GGA) {
                GT* eg = reinterpret_cast<GT*>(S.e[r] + kECols * 128);
                tc::bulk_g2s(eg, gx + off, gbytes, &S.e_full[r]);
                tc::bulk_g2s(eg + kECols * 128, gy + off, gbytes, &S.e_full[r]);
                tc::bulk_g2s(eg + 2 * kECols * 128, gz + off, gbytes, &S.e_full[r]);
              }
            }
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 8) {
    if (lane == 0) {  // MMA issuer
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
            const int s = it % kDStages;
            if (!tc::mbar_wait(&S.full[s], (it / kDStages) & 1)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
            oz_mma_fused<kN>(tbase + b * kAccCols, tc::smem_u32(S.a[s]), kBlkA, 256, tc::smem_u32(S.b[s]), k == 0);
            tc::mma_commit(&S.empty[s]);
          }
          tc::mma_commit(&S.acc_full[b]);
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == 9) {
    if (lane == 0) {  // operand producer: per K step the phi digits (A) and the gathered P digits (B)
      int it = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nK = n / 32, nN = (n + kN - 1) / kN;
        const int8_t* asrc = tA + sb * kDigBytesPerSlot;
        const int8_t* bsrc = tB + (b_off[t0 + ti] - b_off[t0]) * kOpB;
        for (int j = 0; j < nN && ok; ++j)
          for (int k = 0; k < nK; ++k, ++it) {
            const int s = it % kDStages;
            if (it >= kDStages && !tc::mbar_wait(&S.empty[s], ((it / kDStages) - 1) & 1)) {
              ok = false;
              break;
            }
            tc::mbar_expect_tx(&S.full[s], kOpA + kOpB);
            tc::bulk_g2s(S.a[s], asrc + (int64_t)k * kOpA, kOpA, &S.full[s]);
            tc::bulk_g2s(S.b[s], bsrc + (int64_t)(j * nK + k) * kOpB, kOpB, &S.full[s]);
          }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp >= 15) {
    // idle: the CTA holds the whole SM
  } else {  // epilogue: point row = 32 (warp & 3) + lane, columns 16 third .. +15 of each slot block
    const int row = (warp & 3) * 32 + lane, third = warp < 8 ? (warp >> 2) : 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16);
    int jj = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
      const int64_t sg = tso[t0 + ti];
      const int64_t sb = sg - s0;
      const int n = (int)(tso[t0 + ti + 1] - sg);
      const int nN = (n + kN - 1) / kN;
      const double rs = pow2(e_pt[ti * 128 + row] + kCombShift);
      double r_acc = 0.0, g_acc[3] = {0.0, 0.0, 0.0};
      for (int j = 0; j < nN && ok; ++j, ++jj) {
        const int b = jj & 1;
        // the P row scale of column lane (< 16) of this warp's third, broadcast below
        const int cl = j * kN + third * 16 + lane;
        const double psl = (lane < 16 && cl < n) ? __ldg(ps + sb + cl) : 0.0;
        if (!tc::mbar_wait_warp(&S.acc_full[b], (jj >> 1) & 1)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        double x[16];
        acc_cols<16>(trow + b * kAccCols + third * 16, x);
        tc::fence_before_sync();
        tc::mbar_arrive(&S.acc_empty[b]);
#pragma unroll
        for (int u = 0; u < kEGroups; ++u) {
          const int e = (jj * kEGroups + u) * kEThirds + third, r = e % kERing;
          if (!tc::mbar_wait(&S.e_full[r], (e / kERing) & 1)) {
            ok = false;
            break;
          }
          const int c0 = j * kN + third * 16 + u * kECols;
          const double* eb = S.e[r];
          const GT* eg = reinterpret_cast<const GT*>(eb + kECols * 128);
#pragma unroll
          for (int v = 0; v < kECols; ++v) {
            const double X = x[u * kECols + v] * (rs * __shfl_sync(0xffffffffu, psl, u * kECols + v));
            if (c0 + v < n) {
              r_acc += X * eb[v * 128 + row];
              if (GGA) {
                g_acc[0] += X * (double)eg[v * 128 + row];
                g_acc[1] += X * (double)eg[(kECols + v) * 128 + row];
                g_acc[2] += X * (double)eg[(2 * kECols + v) * 128 + row];
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
// scale_exp of the largest of the warp's values v >= 0, from exponent fields
// alone: the high word of a non-negative double orders like the value, so the
// warp's largest high word holds the largest exponent field, and for a normal
// maximum field - 1022 is scale_exp's ilogb + 1.  A maximum of 0 (or one
// below the normal range, which no digit can resolve) gives 0.  One integer
// reduction in place of five double shuffles and maxima.
__device__ __forceinline__ int warp_scale_exp(double v) {
  const unsigned m = __reduce_max_sync(0xffffffffu, (unsigned)((unsigned long long)__double_as_longlong(v) >> 32));
  const int field = (int)(m >> 20);
  return field == 0 ? 0 : field - 1022;
}

// Persistent, one CTA per SM.  Warp kZWarps (one thread) streams the chunk's
// phi and grad phi rows through a ring of stages of kZStage slots by bulk
// copies, and each tile's A and B into a double buffer; warps 0 .. kZWarps-1
// take one slot of every stage each (lane = 4 consecutive points), form
// Z = A phi (+ B . grad phi) in FP64, the scales and the digits, and store
// them.  The copies of
// the next stages are in flight while a stage is converted, so the reads run
// at the HBM rate instead of one load latency per slot group.
constexpr int kZWarps = 16;                          // consumer warps, one slot of each stage each
constexpr int kZStage = kZWarps;                     // slots per ring stage
constexpr int kZThreads = kBlock4((kZWarps + 1) * 32);  // + the producer warp; the rest idle
template <bool GGA, typename GT>
struct ZLayout {
  static constexpr int kRing = (GGA && sizeof(GT) == 8) ? 3 : 4;
  static constexpr int kF = kZStage * 128 * 8;                        // phi of a stage
  static constexpr int kG = GGA ? kZStage * 128 * (int)sizeof(GT) : 0;  // one gradient plane of a stage
  static constexpr int kStage = kF + 3 * kG;
  static constexpr int kAB = 4 * 128 * 8;  // A, Bx, By, Bz of a tile
  static constexpr int kBar = kRing * kStage + 2 * kAB;
  static constexpr int kBytes = kBar + (2 * kRing + 4) * 8;
};

template <bool GGA, typename GT>
__global__ void __launch_bounds__(kZThreads, 1) k_sm_zquant(const int64_t* __restrict__ tso, int64_t t0, int64_t nt,
                                                            int64_t s0, const double* __restrict__ phi,
                                                            const GT* __restrict__ gx, const GT* __restrict__ gy,
                                                            const GT* __restrict__ gz, const double* __restrict__ A,
                                                            const double* __restrict__ Bx,
                                                            const double* __restrict__ By,
                                                            const double* __restrict__ Bz, int8_t* __restrict__ tZ,
                                                            int8_t* __restrict__ tF, double* __restrict__ zs,
                                                            double* __restrict__ fs, int* err) {
  using L = ZLayout<GGA, GT>;
  extern __shared__ __align__(128) uint8_t zsm[];
  uint64_t* full = reinterpret_cast<uint64_t*>(zsm + L::kBar);
  uint64_t* empty = full + L::kRing;
  uint64_t* ab_full = empty + L::kRing;
  uint64_t* ab_empty = ab_full + 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int r = 0; r < L::kRing; ++r) {
      tc::mbar_init(&full[r], 1);
      tc::mbar_init(&empty[r], kZWarps);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&ab_full[b], 1);
      tc::mbar_init(&ab_empty[b], kZWarps);
    }
    tc::mbar_fence_init();
  }
  __syncthreads();
  bool ok = true;
  if (warp == kZWarps) {
    if (lane == 0) {  // producer
      int it = 0, tt = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x, ++tt) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int b = tt & 1;
        if (tt >= 2 && !tc::mbar_wait(&ab_empty[b], ((tt >> 1) - 1) & 1)) {
          ok = false;
          break;
        }
        double* ab = reinterpret_cast<double*>(zsm + L::kRing * L::kStage + b * L::kAB);
        tc::mbar_expect_tx(&ab_full[b], (GGA ? 4 : 1) * 1024);
        tc::bulk_g2s(ab, A + ti * 128, 1024, &ab_full[b]);
        if (GGA) {
          tc::bulk_g2s(ab + 128, Bx + ti * 128, 1024, &ab_full[b]);
          tc::bulk_g2s(ab + 256, By + ti * 128, 1024, &ab_full[b]);
          tc::bulk_g2s(ab + 384, Bz + ti * 128, 1024, &ab_full[b]);
        }
        for (int i0 = 0; i0 < n; i0 += kZStage, ++it) {
          const int r = it % L::kRing;
          if (it >= L::kRing && !tc::mbar_wait(&empty[r], ((it / L::kRing) - 1) & 1)) {
            ok = false;
            break;
          }
          const int ns = min(kZStage, n - i0);
          const int64_t o = (sb + i0) * 128;
          uint8_t* st = zsm + r * L::kStage;
          const uint32_t fb = (uint32_t)ns * 128 * 8, gb = (uint32_t)ns * 128 * sizeof(GT);
          tc::mbar_expect_tx(&full[r], fb + (GGA ? 3 * gb : 0));
          tc::bulk_g2s(st, phi + o, fb, &full[r]);
          if (GGA) {
            tc::bulk_g2s(st + L::kF, gx + o, gb, &full[r]);
            tc::bulk_g2s(st + L::kF + L::kG, gy + o, gb, &full[r]);
            tc::bulk_g2s(st + L::kF + 2 * L::kG, gz + o, gb, &full[r]);
          }
        }
      }
      if (!ok) atomicExch(err, 1);
      // the copies still in flight land before the CTA exits
      for (int j = max(0, it - L::kRing); j < it; ++j) tc::mbar_wait(&full[j % L::kRing], (j / L::kRing) & 1);
      for (int j = max(0, tt - 2); j < tt; ++j) tc::mbar_wait(&ab_full[j & 1], (j >> 1) & 1);
    }
  } else if (warp < kZWarps) {
    const int p0 = lane * 4;
    const int kstep = lane >> 3, kin = (lane & 7) * 4;
    int it = 0, tt = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x, ++tt) {
      const int64_t sb = tso[t0 + ti] - s0;
      const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
      const int b = tt & 1;
      if (!tc::mbar_wait(&ab_full[b], (tt >> 1) & 1)) {
        ok = false;
        break;
      }
      const double* ab = reinterpret_cast<const double*>(zsm + L::kRing * L::kStage + b * L::kAB);
      double a[4], bv[3][4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = ab[p0 + u];
        if (GGA) {
          bv[0][u] = ab[128 + p0 + u];
          bv[1][u] = ab[256 + p0 + u];
          bv[2][u] = ab[384 + p0 + u];
        }
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&ab_empty[b]);
      const int64_t tile_off = sb * kDigBytesPerSlot;
      for (int i0 = 0; i0 < n && ok; i0 += kZStage, ++it) {
        const int r = it % L::kRing;
        if (!tc::mbar_wait(&full[r], (it / L::kRing) & 1)) {
          ok = false;
          break;
        }
        const uint8_t* st = zsm + r * L::kStage;
        const double* fst = reinterpret_cast<const double*>(st);
        if (i0 + warp < n) {
          const int q = warp, i = i0 + q;
          double f[4], z[4];
          const double2 fa = *reinterpret_cast<const double2*>(fst + q * 128 + p0);
          const double2 fb = *reinterpret_cast<const double2*>(fst + q * 128 + p0 + 2);
          f[0] = fa.x; f[1] = fa.y; f[2] = fb.x; f[3] = fb.y;
          if (GGA) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const GT* g = reinterpret_cast<const GT*>(st + L::kF + c * L::kG) + q * 128 + p0;
              double gv[4];
              if constexpr (sizeof(GT) == 4) {
                const float4 w4 = *reinterpret_cast<const float4*>(g);
                gv[0] = w4.x; gv[1] = w4.y; gv[2] = w4.z; gv[3] = w4.w;
              } else {
                const double2 ga = *reinterpret_cast<const double2*>(g);
                const double2 gb2 = *reinterpret_cast<const double2*>(g + 2);
                gv[0] = ga.x; gv[1] = ga.y; gv[2] = gb2.x; gv[3] = gb2.y;
              }
#pragma unroll
              for (int u = 0; u < 4; ++u) z[u] = (c == 0 ? 0.0 : z[u]) + bv[c][u] * gv[u];
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) z[u] = GGA ? z[u] + a[u] * f[u] : a[u] * f[u];
          const int ez = warp_scale_exp(fmax(fmax(fabs(z[0]), fabs(z[1])), fmax(fabs(z[2]), fabs(z[3]))));
          const int ef = warp_scale_exp(fmax(fmax(fabs(f[0]), fabs(f[1])), fmax(fabs(f[2]), fabs(f[3]))));
          if (lane == 0) {
            zs[sb + i] = pow2(ez);
            fs[sb + i] = pow2(ef + kCombShift);
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
          const int64_t kb = tile_off + (int64_t)kstep * n * (32 * kSlices);
#pragma unroll
          for (int sl = 0; sl < kSlices; ++sl) {
            *reinterpret_cast<uint32_t*>(tF + kb + ilv_off(i, kin, sl)) = wf[sl];
            *reinterpret_cast<uint32_t*>(tZ + kb + (int64_t)sl * n * 32 + blk_off(i, kin)) = wz[sl];
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[r]);
      }
    }
    if (!ok) atomicExch(err, 1);
  }
}

// ---------------------------------------------------------------------------
// H[S_t, S_t] += Z_t^T phi_t, scatter-added into V with FP64 atomics (LDA:
// fn_i <= fn_j only, H is symmetric; GGA: the whole square, V = H + H^T when
// packing, the ham + ham^T of modules/xc_hamiltonian.f90:1559-1566).
// Computed as D = phi_J Z_I^T: the 128 TMEM lanes are columns j of H, so the
// 32 atomics of a warp instruction run along one row of V (consecutive
// functions, few sectors).  Pairs of 128-slot blocks J (A, phi) and 48-slot
// blocks I (B, Z); K = the tile's 128 points in 4 steps; each A block is one
// copy of whole 8-slot groups and stays resident for its 48-slot blocks.
// Persistent like k_sm_density.
// ---------------------------------------------------------------------------
constexpr int kVStages = 8;
struct VSmem {
  alignas(1024) int8_t a[2][4][kOpA];      // phi digits of a 128-slot block, all 4 K steps, double-buffered
  alignas(1024) int8_t b[kVStages][kOpB];  // Z digits of a 48-slot block, one K step
  uint64_t a_full[2], a_empty[2];
  uint64_t full[kVStages];
  uint64_t empty[kVStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint32_t tslot;
};
// warps 0-15 epilogue (four per TMEM lane quarter, 12 columns of each 48-slot
// block each), 16 MMA, 17 producer, 18-19 idle
constexpr int kVEpiWarps = 16;
constexpr int kVThreads = (kVEpiWarps + 4) * 32;

// LDA keeps j >= i: the last 48-slot row block I of column block J
__device__ __forceinline__ int last_I(int J, int nI, bool all) { return all ? nI : min(nI, (kM * J + kM - 1) / kN + 1); }

template <bool GGA, bool SET>
__global__ void __launch_bounds__(kVThreads, 1)
    k_sm_vpot(const int64_t* __restrict__ tso, const int* __restrict__ slot_fn, int64_t t0, int64_t nt, int64_t s0,
              const int8_t* __restrict__ tF, const int8_t* __restrict__ tZ, const double* __restrict__ fs,
              const double* __restrict__ zs, double* __restrict__ V, int64_t ldv, int* err,
              const int* __restrict__ tile_mol, const SetMolDev* __restrict__ mols) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  VSmem& S = *reinterpret_cast<VSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(&S.tslot, 512);
  if (tid == 0) {
    for (int q = 0; q < 2; ++q) {
      tc::mbar_init(&S.a_full[q], 1);
      tc::mbar_init(&S.a_empty[q], 1);
    }
    for (int s = 0; s < kVStages; ++s) {
      tc::mbar_init(&S.full[s], 1);
      tc::mbar_init(&S.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&S.acc_full[b], 1);
      tc::mbar_init(&S.acc_empty[b], 32 * kVEpiWarps);
    }
    tc::mbar_fence_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = S.tslot;
  bool ok = true;
  if (warp == kVEpiWarps + 1) {
    if (lane == 0) {  // producer: the phi block of each J once, the Z block of each (J, I) pair per K step
      int it = 0, ia = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int64_t sb = tso[t0 + ti] - s0;
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nJ = (n + kM - 1) / kM, nI = (n + kN - 1) / kN;
        const int8_t* fsrc = tF + sb * kDigBytesPerSlot;
        const int8_t* zsrc = tZ + sb * kDigBytesPerSlot;
        const int64_t kblk = (int64_t)n * 32 * kSlices;  // bytes of one K step of the tile
        for (int J = 0; J < nJ && ok; ++J, ++ia) {
          const int qa = ia & 1;
          if (ia >= 2 && !tc::mbar_wait(&S.a_empty[qa], ((ia >> 1) - 1) & 1)) {
            ok = false;
            break;
          }
          tc::mbar_expect_tx(&S.a_full[qa], 4 * kOpA);
          for (int k = 0; k < 4; ++k)
            tc::bulk_g2s(S.a[qa][k], fsrc + k * kblk + (int64_t)J * (kM / 8) * kIlvGroup, kOpA, &S.a_full[qa]);
          for (int I = 0; I < last_I(J, nI, GGA) && ok; ++I)
            for (int k = 0; k < 4; ++k, ++it) {
              const int s = it % kVStages;
              if (it >= kVStages && !tc::mbar_wait(&S.empty[s], ((it / kVStages) - 1) & 1)) {
                ok = false;
                break;
              }
              tc::mbar_expect_tx(&S.full[s], kOpB);
              for (int sl = 0; sl < kSlices; ++sl)
                tc::bulk_g2s(S.b[s] + sl * kBlkB, zsrc + k * kblk + (int64_t)sl * n * 32 + (int64_t)I * kN * 32, kBlkB,
                             &S.full[s]);
            }
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp == kVEpiWarps) {
    if (lane == 0) {  // MMA issuer
      int it = 0, pp = 0, ia = 0;
      for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
        const int n = (int)(tso[t0 + ti + 1] - tso[t0 + ti]);
        const int nJ = (n + kM - 1) / kM, nI = (n + kN - 1) / kN;
        for (int J = 0; J < nJ && ok; ++J, ++ia) {
          const int qa = ia & 1;
          if (!tc::mbar_wait(&S.a_full[qa], (ia >> 1) & 1)) {
            ok = false;
            break;
          }
          for (int I = 0; I < last_I(J, nI, GGA) && ok; ++I, ++pp) {
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
              oz_mma_fused<kN>(tbase + b * kAccCols, tc::smem_u32(S.a[qa][k]), 256, kIlvGroup, tc::smem_u32(S.b[s]),
                               k == 0);
              tc::mma_commit(&S.empty[s]);
            }
            tc::mma_commit(&S.acc_full[b]);
          }
          tc::mma_commit(&S.a_empty[qa]);
        }
      }
      if (!ok) atomicExch(err, 1);
    }
  } else if (warp > kVEpiWarps + 1) {
    // idle: the CTA holds the whole SM
  } else {  // epilogue: column j = 128 J + 32 (warp & 3) + lane of H, rows 12 part .. +11 of each 48-slot block
    const int part = warp >> 2;
    const uint32_t trow = tbase + ((uint32_t)((warp & 3) * 32) << 16);
    int pp = 0;
    for (int64_t ti = blockIdx.x; ti < nt && ok; ti += gridDim.x) {
      const int64_t sg = tso[t0 + ti];
      const int64_t sb = sg - s0;
      const int n = (int)(tso[t0 + ti + 1] - sg);
      const int nJ = (n + kM - 1) / kM, nI = (n + kN - 1) / kN;
      const int* sfn = slot_fn + sg;
      double* Vt = V;  // this tile's potential matrix (a set: its context's)
      int64_t ldt = ldv;
      if (SET) {
        const SetMolDev& M = mols[tile_mol[t0 + ti]];
        Vt = M.V;
        ldt = M.ldv;
      }
      for (int J = 0; J < nJ && ok; ++J) {
        const int j = J * kM + (warp & 3) * 32 + lane;
        const int fj = j < n ? __ldg(sfn + j) : -1;
        const double fsj = j < n ? __ldg(fs + sb + j) : 0.0;
        for (int I = 0; I < last_I(J, nI, GGA); ++I, ++pp) {
          const int b = pp & 1;
          // row i of lane (< 12) of this warp's 12: its function and scale, broadcast below
          const int il = I * kN + part * 12 + lane;
          const int fil = (lane < 12 && il < n) ? __ldg(sfn + il) : -1;
          const double zsl = (lane < 12 && il < n) ? __ldg(zs + sb + il) : 0.0;
          if (!tc::mbar_wait_warp(&S.acc_full[b], (pp >> 1) & 1)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          double x[12];
          acc_cols<8>(trow + b * kAccCols + part * 12, x);
          acc_cols<4>(trow + b * kAccCols + part * 12 + 8, x + 8);
          tc::fence_before_sync();
          tc::mbar_arrive(&S.acc_empty[b]);
#pragma unroll
          for (int c = 0; c < 12; ++c) {
            const int fi = __shfl_sync(0xffffffffu, fil, c);
            const double zsc = __shfl_sync(0xffffffffu, zsl, c);
            if (fj >= 0 && fi >= 0 && (GGA || fj >= fi)) atomicAdd(Vt + (int64_t)fi * ldt + fj, x[c] * (fsj * zsc));
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
int64_t screen_mixed_bstages(int64_t n) { return ((n + kN - 1) / kN) * (n / 32); }
int64_t screen_mixed_bytes_per_bstage() { return kOpB; }
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
  m->nspin = in.nspin;
  cudaError_t e = cudaSuccess;
  const size_t dig = (size_t)in.chunk_slots * kDigBytesPerSlot;
  const size_t dig_a = (size_t)std::max(in.chunk_slots, in.resident_slots) * kDigBytesPerSlot;
  for (int s = 0; s < in.nspin; ++s) {
    if (e == cudaSuccess) e = sm_alloc(m, &m->P8[s], (size_t)in.nbas * in.nbas);
    if (e == cudaSuccess) e = sm_alloc(m, &m->e_P[s], (size_t)in.nbas);
  }
  if (e == cudaSuccess) e = sm_alloc(m, &m->tA, dig_a);
  if (e == cudaSuccess) e = sm_alloc(m, &m->tB, (size_t)in.chunk_bstages * kOpB);
  m->b_off = in.b_off;
  if (e == cudaSuccess) e = sm_alloc(m, &m->tZ, dig);
  if (e == cudaSuccess) e = sm_alloc(m, &m->tF, dig);
  if (e == cudaSuccess) e = sm_alloc(m, &m->e_pt, (size_t)std::max(in.chunk_tiles, in.resident_tiles) * 128);
  if (e == cudaSuccess) e = sm_alloc(m, &m->zs, (size_t)in.chunk_slots);
  if (e == cudaSuccess) e = sm_alloc(m, &m->fs, (size_t)in.chunk_slots);
  if (e == cudaSuccess) e = sm_alloc(m, &m->ps, (size_t)in.chunk_slots);
  if (e == cudaSuccess) e = sm_alloc(m, &m->err, 1);
  // the slack rows after a chunk's last slot are read (never used) by whole-block copies
  if (e == cudaSuccess) e = cudaMemset(m->tA, 0, dig_a);
  if (e == cudaSuccess) e = cudaMemset(m->tZ, 0, dig);
  if (e == cudaSuccess) e = cudaMemset(m->tF, 0, dig);
  if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
  if (e != cudaSuccess) {
    err = std::string("screened mixed-precision buffers: ") + cudaGetErrorString(e);
    screen_mixed_destroy(m);
    return e == cudaErrorMemoryAllocation ? PGXC_ENOMEM : PGXC_ECUDA;
  }
  static_assert(sizeof(DensSmem) <= tc::kWholeSmSmem && sizeof(VSmem) <= tc::kWholeSmSmem, "smem");
  static_assert(ZLayout<true, double>::kBytes <= tc::kWholeSmSmem && ZLayout<true, float>::kBytes <= tc::kWholeSmSmem,
                "smem");
  const int dsm = tc::kWholeSmSmem;
  raise_smem_limit(k_sm_gather_B, 4 * in.max_n);
  cudaFuncSetAttribute(k_sm_zquant<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       ZLayout<true, double>::kBytes);
  cudaFuncSetAttribute(k_sm_zquant<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       ZLayout<true, float>::kBytes);
  cudaFuncSetAttribute(k_sm_zquant<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       ZLayout<false, double>::kBytes);
  cudaFuncSetAttribute(k_sm_zquant<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       ZLayout<false, float>::kBytes);
  cudaFuncSetAttribute(k_sm_density<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_density<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_density<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_density<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm);
  cudaFuncSetAttribute(k_sm_vpot<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kWholeSmSmem);
  cudaFuncSetAttribute(k_sm_vpot<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kWholeSmSmem);
  cudaFuncSetAttribute(k_sm_vpot<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kWholeSmSmem);
  e = cudaFuncSetAttribute(k_sm_vpot<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kWholeSmSmem);
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

int screen_mixed_prepare(ScreenMixed* m, const double* P, int64_t ldc, int spin, cudaStream_t st) {
  k_sm_rowexp_P<<<(unsigned)m->nbas, 256, 0, st>>>(P, ldc, m->nbas, m->e_P[spin]);
  const unsigned nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((m->nbas * m->nbas + 255) / 256, 148 * 16));
  k_sm_quant_P<<<nb, 256, 0, st>>>(P, ldc, m->nbas, m->e_P[spin], m->P8[spin]);
  return 2;
}

int screen_mixed_basis(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                       const double* phi, const unsigned long long* pmax, int64_t so, int64_t to, cudaStream_t st,
                       const int* tile_mol, const SetMolDev* mols) {
  k_sm_quant_pts<<<(unsigned)nt, 128, 0, st>>>(tso, t0, s0, phi, pmax, m->e_pt + to * 128,
                                              m->tA + so * kDigBytesPerSlot);
  return 1 + screen_mixed_gather(m, tso, slot_fn, t0, nt, s0, 0, st, tile_mol, mols);
}

void screen_mixed_set_gga(ScreenMixed* m, bool gga) { m->gga = gga; }

int screen_mixed_gather(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                        int spin, cudaStream_t st, const int* tile_mol, const SetMolDev* mols) {
  k_sm_gather_B<<<dim3((unsigned)nt, kGatherSplit), kBlock4(192), 4 * m->max_n, st>>>(
      tso, slot_fn, m->b_off, t0, s0, m->P8[spin], m->e_P[spin], m->nbas, m->tB, m->ps, tile_mol, mols);
  return 1;
}

namespace {

template <typename GT>
int mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                  const double* phi, const GT* gx, const GT* gy, const GT* gz, double* rho, double* grx, double* gry,
                  double* grz, int64_t so, int64_t to, cudaStream_t st) {
  const int8_t* tA = m->tA + so * kDigBytesPerSlot;
  const int* e_pt = m->e_pt + to * 128;
  cudaMemsetAsync(rho, 0, sizeof(double) * nt * 128, st);
  if (m->gga) {
    cudaMemsetAsync(grx, 0, sizeof(double) * nt * 128, st);
    cudaMemsetAsync(gry, 0, sizeof(double) * nt * 128, st);
    cudaMemsetAsync(grz, 0, sizeof(double) * nt * 128, st);
  }
  const unsigned grid = (unsigned)std::min<int64_t>(nt, m->nsm);
  const int smem = tc::kWholeSmSmem;
  if (m->gga)
    k_sm_density<true, GT><<<grid, kDensThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, tA, e_pt, m->tB, m->b_off,
                                                             m->ps, phi, gx, gy, gz, rho, grx, gry, grz, m->err);
  else
    k_sm_density<false, GT><<<grid, kDensThreads, smem, st>>>(tso, slot_fn, t0, nt, s0, tA, e_pt, m->tB, m->b_off,
                                                              m->ps, phi, nullptr, nullptr, nullptr, rho, nullptr,
                                                              nullptr, nullptr, m->err);
  return 1;
}

template <typename GT>
int mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                    const double* phi, const GT* gx, const GT* gy, const GT* gz, const double* A, const double* Bx,
                    const double* By, const double* Bz, double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0,
                    cudaEvent_t k1, const int* tile_mol, const SetMolDev* mols) {
  const unsigned zgrid = (unsigned)std::min<int64_t>(nt, m->nsm);
  if (m->gga)
    k_sm_zquant<true, GT><<<zgrid, kZThreads, ZLayout<true, GT>::kBytes, st>>>(
        tso, t0, nt, s0, phi, gx, gy, gz, A, Bx, By, Bz, m->tZ, m->tF, m->zs, m->fs, m->err);
  else
    k_sm_zquant<false, GT><<<zgrid, kZThreads, ZLayout<false, GT>::kBytes, st>>>(
        tso, t0, nt, s0, phi, nullptr, nullptr, nullptr, A, nullptr, nullptr, nullptr, m->tZ, m->tF, m->zs, m->fs,
        m->err);
  if (k0) cudaEventRecord(k0, st);
  const unsigned grid = (unsigned)std::min<int64_t>(nt, m->nsm);
  auto launch = [&](auto kern) {
    kern<<<grid, kVThreads, tc::kWholeSmSmem, st>>>(tso, slot_fn, t0, nt, s0, m->tF, m->tZ, m->fs, m->zs, V, ldv, m->err,
                                                   tile_mol, mols);
  };
  if (m->gga) {
    if (tile_mol) launch(k_sm_vpot<true, true>);
    else launch(k_sm_vpot<true, false>);
  } else {
    if (tile_mol) launch(k_sm_vpot<false, true>);
    else launch(k_sm_vpot<false, false>);
  }
  if (k1) cudaEventRecord(k1, st);
  return 2;
}

}  // namespace

int screen_mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                         const double* phi, const double* gx, const double* gy, const double* gz, double* rho,
                         double* grx, double* gry, double* grz, int64_t so, int64_t to, cudaStream_t st) {
  return mixed_density<double>(m, tso, slot_fn, t0, nt, s0, phi, gx, gy, gz, rho, grx, gry, grz, so, to, st);
}
int screen_mixed_density(ScreenMixed* m, const int64_t* tso, const int* slot_fn, int64_t t0, int64_t nt, int64_t s0,
                         const double* phi, const float* gx, const float* gy, const float* gz, double* rho,
                         double* grx, double* gry, double* grz, int64_t so, int64_t to, cudaStream_t st) {
  return mixed_density<float>(m, tso, slot_fn, t0, nt, s0, phi, gx, gy, gz, rho, grx, gry, grz, so, to, st);
}

int screen_mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, const int* slot_tile, int64_t t0,
                           int64_t nt, int64_t s0, int64_t ns, const double* phi, const double* gx, const double* gy,
                           const double* gz, const double* A, const double* Bx, const double* By, const double* Bz,
                           double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1,
                           const int* tile_mol, const SetMolDev* mols) {
  (void)slot_tile;
  (void)ns;
  return mixed_potential<double>(m, tso, slot_fn, t0, nt, s0, phi, gx, gy, gz, A, Bx, By, Bz, V, ldv, st, k0, k1,
                                 tile_mol, mols);
}
int screen_mixed_potential(ScreenMixed* m, const int64_t* tso, const int* slot_fn, const int* slot_tile, int64_t t0,
                           int64_t nt, int64_t s0, int64_t ns, const double* phi, const float* gx, const float* gy,
                           const float* gz, const double* A, const double* Bx, const double* By, const double* Bz,
                           double* V, int64_t ldv, cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1,
                           const int* tile_mol, const SetMolDev* mols) {
  (void)slot_tile;
  (void)ns;
  return mixed_potential<float>(m, tso, slot_fn, t0, nt, s0, phi, gx, gy, gz, A, Bx, By, Bz, V, ldv, st, k0, k1,
                                tile_mol, mols);
}

void screen_mixed_p8(ScreenMixed* m, int spin, const unsigned long long** P8, const int** e_P) {
  *P8 = m->P8[spin];
  *e_P = m->e_P[spin];
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
